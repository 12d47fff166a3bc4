// fw_syn.cu -- the SyN stage driver (syn.rs:337-445, 776-986) on the device.
//
// One iteration (syn.rs:890-958): warp fixed and moving through F^-1 and affine(M^-1); the CC
// pair (window sums shared by both directions); for several channels the multi-metric
// combination (syn.rs:203-282); Gaussian smoothing of both gradients with the max |u/sp| fused;
// F <- F + (step / max) u(x + F) (scale fused into the composition, done in place because every
// voxel reads only its own F); optional total-field smoothing; the inversion pair
// F^-1 = invert(F, init F^-1), F = invert(F^-1, init F) in place; then the energy enters the
// window convergence monitor (convergence.rs:47-126).
//
// Graph design: every buffer of a level is allocated once, so the kernel sequence of an
// iteration is the same every time. The whole level is captured as ONE CUDA graph: an outer
// WHILE node whose body is the iteration, with each of the four inversions an inner WHILE node
// whose condition the inversion step's last block sets (no host read-back inside the loop); the
// iteration's first kernel sets the four loops' states and conditions and clears the update
// maxima. A
// single-thread record kernel at the end of the body runs the convergence monitor on the device,
// writes the iteration record and sets the outer condition. The host launches one graph and
// reads the records back once per level.
#include <cuda_runtime.h>

#include <cfloat>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fw_internal.cuh"
#include "fw_syn_state.cuh"

namespace fw {

namespace {

// A level whose run is enqueued behind a failed one (the status is kept from level to level)
// runs no iteration: the host reads the status once, after the last level.
__global__ void k_syn_level_init(SynDev* s, int level, int limit,
                                 cudaGraphConditionalHandle handle, int use_handle) {
    const int run = syn_level_begin(s, level, limit);
    if (use_handle) cudaGraphSetConditional(handle, run ? 1u : 0u);
}

__global__ void k_syn_record(SynDev* s, const double* __restrict__ cc,
                             const unsigned int* __restrict__ max_bits,
                             const InvState* __restrict__ inv, fw_syn_iteration* trace,
                             int trace_cap, const volatile int* cancel,
                             cudaGraphConditionalHandle handle, int use_handle) {
    pdl_wait();
    const int more = syn_record_step(s, cc, max_bits, inv, trace, trace_cap, cancel);
    if (use_handle) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// acc += (w / |x|) x when |x| > eps (syn.rs:233-240), |x|^2 read from the device.
__global__ void k_axpy_norm(float4* __restrict__ acc, const float4* __restrict__ x, long long n4,
                            const double* __restrict__ nsq, double w) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n4) return;
    double mag = sqrt(*nsq);
    if (!(mag > DBL_EPSILON)) return;
    float a = (float)(w / mag);
    float4 v = acc[l], u = x[l];
    v.x = fmaf(a, u.x, v.x);
    v.y = fmaf(a, u.y, v.y);
    v.z = fmaf(a, u.z, v.z);
    v.w = fmaf(a, u.w, v.w);
    acc[l] = v;
}

// acc *= sum_c |d_c| / C (syn.rs:259-263); `which` selects |dF|^2 (1) or |dM|^2 (2).
__global__ void k_scale_norms(float4* __restrict__ acc, long long n4, const double* __restrict__ cc,
                              int channels, int which) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n4) return;
    double tot = 0.0;
    for (int c = 0; c < channels; ++c) tot += sqrt(cc[CC_STRIDE * c + which]);
    float s = (float)(tot / channels);
    float4 v = acc[l];
    v.x *= s;
    v.y *= s;
    v.z *= s;
    v.w *= s;
    acc[l] = v;
}

struct Level {
    HostGrid grid;
    int channels = 1;
    fw_field *F = nullptr, *Fi = nullptr, *M = nullptr, *Mi = nullptr;
    std::vector<fw_image*> fmid, mmid;
    fw_field *dF = nullptr, *dM = nullptr;      // raw CC derivatives
    fw_field *accF = nullptr, *accM = nullptr;  // multichannel combination
    fw_field *sF = nullptr, *sM = nullptr;      // smoothed updates
    fw_field* T = nullptr;                      // total-field smoothing
    fw_field* R = nullptr;                      // inversion residual of the last measurement
    const fw_image* fmask = nullptr;            // recipe masks on their own grids (or none)
    const fw_image* mmask = nullptr;
    fw_image* fvalid = nullptr;                 // each given mask resolved on the level grid
    fw_image* mvalid = nullptr;
    fw_image* valid = nullptr;                  // inside both (the CC pairs' voxels)
    fw_dense_mi* mi = nullptr;                  // scratch of the Mattes pairs
    const fw_field* prior = nullptr;            // earlier SyN stages' collapsed field (or none)
};

void free_level_work(Level& L) {
    for (auto* im : L.fmid) fw_image_free(im);
    for (auto* im : L.mmid) fw_image_free(im);
    L.fmid.clear();
    L.mmid.clear();
    fw_image_free(L.valid);
    fw_image_free(L.fvalid);
    fw_image_free(L.mvalid);
    L.valid = L.fvalid = L.mvalid = nullptr;
    dense_mi_free(L.mi);
    L.mi = nullptr;
    fw_field* fs[] = {L.dF, L.dM, L.accF, L.accM, L.sF, L.sM, L.T, L.R};
    for (auto* f : fs) fw_field_free(f);
    L.dF = L.dM = L.accF = L.accM = L.sF = L.sM = L.T = L.R = nullptr;
}

int alloc_level_work(fw_ctx* ctx, const fw_syn_recipe* r, Level& L) {
    for (int c = 0; c < L.channels; ++c) {
        fw_image *a, *b;
        FW_TRY(new_image(ctx, L.grid, &a));
        L.fmid.push_back(a);
        FW_TRY(new_image(ctx, L.grid, &b));
        L.mmid.push_back(b);
    }
    FW_TRY(new_field(ctx, L.grid, &L.dF));
    FW_TRY(new_field(ctx, L.grid, &L.dM));
    FW_TRY(new_field(ctx, L.grid, &L.R));
    if (L.channels > 1) {
        FW_TRY(new_field(ctx, L.grid, &L.accF));
        FW_TRY(new_field(ctx, L.grid, &L.accM));
    }
    if (r->update_field_variance > 0.0) {
        FW_TRY(new_field(ctx, L.grid, &L.sF));
        FW_TRY(new_field(ctx, L.grid, &L.sM));
    }
    if (r->total_field_variance > 0.0) FW_TRY(new_field(ctx, L.grid, &L.T));
    if (L.fmask) FW_TRY(new_image(ctx, L.grid, &L.fvalid));
    if (L.mmask) FW_TRY(new_image(ctx, L.grid, &L.mvalid));
    if (L.fmask && L.mmask) FW_TRY(new_image(ctx, L.grid, &L.valid));
    bool mattes = false;
    for (int c = 0; c < L.channels; ++c) mattes = mattes || r->channel_metrics[c] == FW_METRIC_MATTES;
    if (mattes) FW_TRY(dense_mi_create(ctx, r->mi_bins, L.grid.count(), &L.mi));
    return 0;
}

// Device scalars of a run.
struct RunDev {
    SynDev* syn;
    double* cc;              // [channels][CC_STRIDE]
    unsigned int* max_bits;  // [2]
    InvState* inv;           // [4]
    fw_syn_iteration* trace;
    int trace_cap;
};

const fw_invert_params kSynInvert = {20, 0.001, 0.1, 1};

}  // namespace

// Adds a WHILE node on an existing handle at the capture position of `s`.
int add_while_node(cudaStream_t s, cudaGraphConditionalHandle handle, cudaGraph_t* body) {
    cudaStreamCaptureStatus status;
    cudaGraph_t g;
    const cudaGraphNode_t* deps;
    size_t ndeps;
    FW_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, &g, &deps, &ndeps));
    FW_CHECK(status == cudaStreamCaptureStatusActive, "graph capture is not active");
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    FW_CUDA(cudaGraphAddNode(&node, g, deps, ndeps, &p));
    *body = p.conditional.phGraph_out[0];
    FW_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return 0;
}

namespace {

// One inversion: in graph mode a WHILE node around the body kernels on `h` (the iteration's first
// kernel set the loop's state and condition); in direct mode its init kernel and a host loop.
int enqueue_invert(fw_ctx* ctx, bool graph, const fw_field* field, fw_field* inverse,
                   fw_field* res, InvState* st, cudaGraphConditionalHandle h) {
    if (!graph) {
        FW_TRY(enqueue_inversion_prefix(ctx, field, inverse, res, kSynInvert, st, 0, 0));
        InvState hs;
        for (int body = 0; body < kSynInvert.max_iterations; ++body) {
            FW_TRY(enqueue_inversion_body(ctx, field, inverse, res, st, 0, 0));
            FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, st, sizeof(InvState), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            FW_TRY(sync(ctx));
            std::memcpy(&hs, ctx->h_pinned, sizeof(hs));
            if (!hs.go) break;
        }
        return 0;
    }
    FW_CHECK(res->grid.same(inverse->grid) && res->ps == inverse->ps,
             "invert: the residual buffer does not match the inverse");
    FW_TRY(inversion_scratch(ctx, field));
    cudaStreamCaptureStatus status;
    cudaGraph_t g;
    const cudaGraphNode_t* deps;
    size_t ndeps;
    FW_CUDA(cudaStreamGetCaptureInfo(ctx->stream, &status, nullptr, &g, &deps, &ndeps));
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    FW_CUDA(cudaGraphAddNode(&node, g, deps, ndeps, &p));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    FW_CUDA(cudaStreamUpdateCaptureDependencies(ctx->stream, &node, 1,
                                                cudaStreamSetCaptureDependencies));
    // capture the body on the auxiliary stream
    cudaStream_t main = ctx->stream;
    FW_CUDA(cudaStreamBeginCaptureToGraph(ctx->aux, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
    ctx->stream = ctx->aux;
    int rc = enqueue_inversion_body(ctx, field, inverse, res, st, h, 1);
    ctx->stream = main;
    cudaGraph_t out;
    cudaError_t e = cudaStreamEndCapture(ctx->aux, &out);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "inversion body capture");
    return 0;
}

unsigned int blocks256(long long n) { return (unsigned int)((n + 255) / 256); }

// The kernels of one iteration (syn.rs:890-958) on ctx->stream.
int enqueue_iteration(fw_ctx* ctx, bool graph, const fw_syn_recipe* r, Level& L,
                      const std::vector<const fw_image*>& fs,
                      const std::vector<const fw_image*>& ms, const fw_affine* initial,
                      const RunDev& d) {
    const int C = L.channels;
    // graph mode: one kernel begins the iteration -- the update maxima cleared, the four
    // inversions' states and WHILE conditions set (their handles live in the graph being
    // captured); direct mode: a memset, and each inversion's init kernel
    cudaGraphConditionalHandle hinv[4] = {0, 0, 0, 0};
    if (graph) {
        cudaStreamCaptureStatus status;
        cudaGraph_t g;
        FW_CUDA(cudaStreamGetCaptureInfo(ctx->stream, &status, nullptr, &g, nullptr, nullptr));
        for (auto& h : hinv) FW_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
        FW_TRY(enqueue_inversion_inits(ctx, d.inv, 4, kSynInvert, hinv, d.max_bits, 2));
    } else {
        FW_CUDA(cudaMemsetAsync(d.max_bits, 0, 2 * sizeof(unsigned int), ctx->stream));
    }
    if (C > 1) {
        FW_CUDA(cudaMemsetAsync(L.accF->d, 0, L.accF->bytes, ctx->stream));
        FW_CUDA(cudaMemsetAsync(L.accM->d, 0, L.accM->bytes, ctx->stream));
    }
    double wsum = 0.0;
    for (int c = 0; c < C; ++c) wsum += r->channel_weights[c];
    const long long n4 = 3 * L.dF->ps / 4;
    // syn.rs:496-580: each given mask resolved on the level grid (nearest voxel, half up), the
    // fixed one through F^-1 and the moving one through affine(M^-1); CC takes the voxels inside
    // both, a Mattes pair each mask on its own
    if (L.fmask)
        FW_TRY(launch_warp(ctx, L.fmask, L.Fi, nullptr, nullptr, L.fvalid->d, true, nullptr));
    if (L.mmask)
        FW_TRY(launch_warp(ctx, L.mmask, L.Mi, L.prior, initial, L.mvalid->d, true, nullptr));
    const fw_image* valid = L.fvalid ? L.fvalid : L.mvalid;
    if (L.fvalid && L.mvalid) {
        FW_TRY(launch_image_product(ctx, L.fvalid, L.mvalid, L.valid));
        valid = L.valid;
    }
    for (int c = 0; c < C; ++c) {
        FW_TRY(launch_warp(ctx, fs[c], L.Fi, nullptr, nullptr, L.fmid[c]->d, false, nullptr));
        FW_TRY(launch_warp(ctx, ms[c], L.Mi, L.prior, initial, L.mmid[c]->d, false, nullptr));
        if (r->channel_metrics[c] == FW_METRIC_MATTES)
            FW_TRY(enqueue_dense_mi_pair(ctx, L.fmid[c], L.mmid[c], L.fvalid, L.mvalid, L.dF,
                                         L.dM, L.mi, d.cc + CC_STRIDE * c));
        else
            FW_TRY(launch_cc_pair_impl(ctx, L.fmid[c], L.mmid[c], r->cc_radius, L.dF, L.dM,
                                       d.cc + CC_STRIDE * c, C > 1 ? 1 : 0, valid));
        if (C > 1) {
            double wn = r->channel_weights[c] / wsum;
            k_axpy_norm<<<blocks256(n4), 256, 0, ctx->stream>>>((float4*)L.accF->d,
                                                                (const float4*)L.dF->d, n4,
                                                                d.cc + CC_STRIDE * c + 1, wn);
            FW_TRY(check_launch(ctx, "k_axpy_norm"));
            k_axpy_norm<<<blocks256(n4), 256, 0, ctx->stream>>>((float4*)L.accM->d,
                                                                (const float4*)L.dM->d, n4,
                                                                d.cc + CC_STRIDE * c + 2, wn);
            FW_TRY(check_launch(ctx, "k_axpy_norm"));
        }
    }
    fw_field* gF = L.dF;
    fw_field* gM = L.dM;
    if (C > 1) {
        k_scale_norms<<<blocks256(n4), 256, 0, ctx->stream>>>((float4*)L.accF->d, n4, d.cc, C, 1);
        FW_TRY(check_launch(ctx, "k_scale_norms"));
        k_scale_norms<<<blocks256(n4), 256, 0, ctx->stream>>>((float4*)L.accM->d, n4, d.cc, C, 2);
        FW_TRY(check_launch(ctx, "k_scale_norms"));
        gF = L.accF;
        gM = L.accM;
    }
    // update_total_field for both sides (syn.rs:422-445), one side after the other: smooth the
    // update (variance in voxels^2) with its max |u/sp| fused; F <- F + (step / max) u(x + F) in
    // place; optional total-field smoothing; the inversion pair. The sides only share scratch
    // (the residual field R), so running them in turn gives the reference's fields.
    struct Side {
        fw_field* g;  // raw update (CC derivative or channel combination)
        fw_field* s;  // smoothed update
        fw_field* field;
        fw_field* inverse;
        unsigned int* max;
        InvState* st;
        const cudaGraphConditionalHandle* h;
    } sides[2] = {{gF, L.sF, L.F, L.Fi, d.max_bits, d.inv, hinv},
                  {gM, L.sM, L.M, L.Mi, d.max_bits + 1, d.inv + 2, hinv + 2}};
    for (auto& s : sides) {
        const fw_field* u = s.g;
        if (r->update_field_variance > 0.0) {
            FW_TRY(launch_smooth(ctx, s.g, s.s, r->update_field_variance, s.max, L.R));
            u = s.s;
        } else {
            FW_TRY(launch_max_norm(ctx, s.g, s.max));
        }
        // compose in place: every voxel reads its own field value and the update elsewhere
        FW_TRY(launch_compose(ctx, u, s.field, s.field, s.max, r->gradient_step));
        if (r->total_field_variance > 0.0) {
            FW_TRY(launch_smooth(ctx, s.field, L.T, r->total_field_variance, nullptr, L.R));
            FW_CUDA(cudaMemcpyAsync(s.field->d, L.T->d, s.field->bytes, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
        }
        // inverse = invert(field), then field = invert(inverse)
        FW_TRY(enqueue_invert(ctx, graph, s.field, s.inverse, L.R, s.st, s.h[0]));
        FW_TRY(enqueue_invert(ctx, graph, s.inverse, s.field, L.R, s.st + 1, s.h[1]));
    }
    return 0;
}

int syn_validate(const fw_syn_recipe* r) {
    FW_CHECK(r, "null recipe");
    FW_CHECK(r->levels >= 1 && r->levels <= FW_MAX_LEVELS, "syn recipe: no levels");
    FW_CHECK(r->channels >= 1 && r->channels <= FW_MAX_CHANNELS, "syn recipe: 1..=4 channels");
    double ws = 0.0;
    for (int c = 0; c < r->channels; ++c) {
        FW_CHECK(std::isfinite(r->channel_weights[c]) && r->channel_weights[c] >= 0.0,
                 "syn recipe: channel weights must be non-negative with a positive sum");
        ws += r->channel_weights[c];
    }
    FW_CHECK(ws > DBL_EPSILON, "syn recipe: channel weights must be non-negative with a positive sum");
    for (int l = 0; l < r->levels; ++l) FW_CHECK(r->shrink_factors[l] > 0, "syn recipe: shrink factor 0");
    FW_CHECK(std::isfinite(r->gradient_step) && r->gradient_step > 0.0,
             "syn recipe: gradient step must be positive");
    FW_CHECK(r->cc_radius >= 1 && r->cc_radius <= 8, "syn recipe: CC radius must be in 1..=8");
    FW_CHECK(r->convergence_window >= 1 && r->convergence_window <= MAX_WINDOW,
             "syn recipe: convergence window must be in 1..=64");
    FW_CHECK(std::isfinite(r->update_field_variance) && std::isfinite(r->total_field_variance),
             "syn recipe: variances must be finite");
    bool mattes = false;
    for (int c = 0; c < r->channels; ++c) {
        FW_CHECK(r->channel_metrics[c] == FW_METRIC_CC || r->channel_metrics[c] == FW_METRIC_MATTES,
                 "syn recipe: unknown channel metric");
        mattes = mattes || r->channel_metrics[c] == FW_METRIC_MATTES;
    }
    // recipe.rs:233-238
    FW_CHECK(!mattes || r->mi_bins >= 5, "syn recipe: MI needs at least five histogram bins");
    FW_CHECK(!mattes || r->mi_bins <= 32, "syn recipe: MI bins must be in 5..=32 on this engine");
    return 0;
}

// pyramid.rs:58-93
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

// pyramid.rs:99-129
int shrink_grid(const HostGrid& g, const uint32_t f[3], HostGrid& out) {
    fw_grid o = to_c(g);
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
    auto index_to_point = [](const HostGrid& gg, const double c[3], double p[3]) {
        double s[3] = {c[0] * gg.sp[0], c[1] * gg.sp[1], c[2] * gg.sp[2]};
        for (int r = 0; r < 3; ++r)
            p[r] = gg.org[r] + (gg.dir[r * 3] * s[0] + gg.dir[r * 3 + 1] * s[1] + gg.dir[r * 3 + 2] * s[2]);
    };
    index_to_point(g, ic, ip);
    HostGrid prov;
    FW_TRY(make_grid(&o, prov));
    index_to_point(prov, oc, op);
    for (int a = 0; a < 3; ++a) o.origin[a] = g.org[a] + (ip[a] - op[a]);
    return make_grid(&o, out);
}

int level_grid(const fw_syn_recipe* r, const HostGrid& fixed, int level, HostGrid& out) {
    uint32_t f[3];
    shrink_factors(r->shrink_factors[level], fixed.sp, f);
    return shrink_grid(fixed, f, out);
}

struct RunScratch {
    fw_ctx* ctx = nullptr;
    void* base = nullptr;
    size_t bytes = 0;
    RunDev d{};
    ~RunScratch() {
        if (base) dev_free(ctx, base, bytes);
    }
    int init(fw_ctx* c, int channels, int trace_cap) {
        ctx = c;
        size_t off_syn = 0;
        size_t off_cc = off_syn + ((sizeof(SynDev) + 255) / 256) * 256;
        size_t off_max = off_cc + 256;
        size_t off_inv = off_max + 256;
        size_t off_trace = off_inv + ((4 * sizeof(InvState) + 255) / 256) * 256;
        bytes = off_trace + sizeof(fw_syn_iteration) * (size_t)std::max(trace_cap, 1);
        (void)channels;
        FW_TRY(dev_alloc(ctx, bytes, &base));
        char* b = static_cast<char*>(base);
        d.syn = reinterpret_cast<SynDev*>(b + off_syn);
        d.cc = reinterpret_cast<double*>(b + off_cc);
        d.max_bits = reinterpret_cast<unsigned int*>(b + off_max);
        d.inv = reinterpret_cast<InvState*>(b + off_inv);
        d.trace = reinterpret_cast<fw_syn_iteration*>(b + off_trace);
        d.trace_cap = trace_cap;
        FW_CUDA(cudaMemsetAsync(base, 0, bytes, ctx->stream));
        return 0;
    }
};

int upload_syn_dev(fw_ctx* ctx, const fw_syn_recipe* r, SynDev* d, bool masked) {
    SynDev h;
    std::memset(&h, 0, sizeof(h));
    h.masked = masked ? 1 : 0;
    for (int c = 0; c < r->channels; ++c) h.metric[c] = r->channel_metrics[c];
    h.window = r->convergence_window;
    h.threshold = r->convergence_threshold;
    h.step = r->gradient_step;
    h.channels = r->channels;
    double ws = 0.0;
    for (int c = 0; c < r->channels; ++c) ws += r->channel_weights[c];
    for (int c = 0; c < r->channels; ++c) h.wnorm[c] = r->channel_weights[c] / ws;
    FW_CUDA(cudaMemcpyAsync(d, &h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream));
    return sync(ctx);  // h lives on this stack frame
}

struct GraphGuard {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~GraphGuard() {
        if (e) cudaGraphExecDestroy(e);
        if (g) cudaGraphDestroy(g);
    }
};

// Captures the level's iteration loop as one graph, launches it and waits.
// FASTWARP_SYN_GRAPHS=0 launches the same kernels straight onto the stream, the loops driven by
// the host (one read-back per inversion body and per iteration): for profilers that cannot look
// inside graphs with conditional nodes, and for debugging. The default is the graph.
bool use_graphs() {
    const char* v = std::getenv("FASTWARP_SYN_GRAPHS");
    return !(v && v[0] == '0');
}

// FASTWARP_TRACE=1: host-side phase times of every level on stderr (capture, instantiate, run).
bool tracing() {
    static const bool on = [] {
        const char* v = std::getenv("FASTWARP_TRACE");
        return v && v[0] == '1';
    }();
    return on;
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

int run_level_direct(fw_ctx* ctx, const fw_syn_recipe* r, Level& L,
                     const std::vector<const fw_image*>& fs, const std::vector<const fw_image*>& ms,
                     const fw_affine* initial, const RunDev& d, int level, int limit,
                     fw_syn_iteration* trace_dev_base) {
    k_syn_level_init<<<1, 1, 0, ctx->stream>>>(d.syn, level, limit, 0, 0);
    FW_TRY(check_launch(ctx, "k_syn_level_init"));
    for (int it = 0; it < limit; ++it) {
        if (cancel_requested(ctx)) return fail(FW_ERR_CANCELLED, "registration cancelled");
        FW_TRY(enqueue_iteration(ctx, false, r, L, fs, ms, initial, d));
        k_syn_record<<<1, 1, 0, ctx->stream>>>(d.syn, d.cc, d.max_bits, d.inv, trace_dev_base,
                                              d.trace_cap, ctx->cancel_mapped_dev, 0, 0);
        FW_TRY(check_launch(ctx, "k_syn_record"));
        FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, d.syn, sizeof(SynDev), cudaMemcpyDeviceToHost,
                                ctx->stream));
        FW_TRY(sync(ctx));
        SynDev h;
        std::memcpy(&h, ctx->h_pinned, sizeof(h));
        if (h.converged || h.status) break;
    }
    return 0;
}

int run_level_graph(fw_ctx* ctx, const fw_syn_recipe* r, Level& L,
                    const std::vector<const fw_image*>& fs, const std::vector<const fw_image*>& ms,
                    const fw_affine* initial, const RunDev& d, int level, int limit,
                    fw_syn_iteration* trace_dev_base) {
    GraphGuard G;
    const double t0 = tracing() ? now_ms() : 0.0;
    const uint64_t launches0 = ctx->stats.kernel_launches;  // captured kernels are not launches
    FW_CUDA(cudaGraphCreate(&G.g, 0));
    // the iteration loop's condition: set by the level init (no iteration after a failed level)
    // and then by the record kernel at the end of every iteration
    cudaGraphConditionalHandle h_it = 0;
    FW_CUDA(cudaGraphConditionalHandleCreate(&h_it, G.g, 0, 0));
    FW_CUDA(cudaStreamBeginCaptureToGraph(ctx->stream, G.g, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
    ctx->capturing = true;
    int rc = 0;
    cudaGraph_t body = nullptr;
    k_syn_level_init<<<1, 1, 0, ctx->stream>>>(d.syn, level, limit, h_it, 1);
    rc = check_launch(ctx, "k_syn_level_init");
    if (!rc) rc = add_while_node(ctx->stream, h_it, &body);
    cudaGraph_t top;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &top);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "level graph capture");
    if (!rc) {
        e = cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed);
        if (e != cudaSuccess) rc = cuda_fail(e, "iteration capture");
        if (!rc) {
            rc = enqueue_iteration(ctx, true, r, L, fs, ms, initial, d);
            if (!rc) {
                // the context's cancel flag is read once per iteration: a cancel stops the
                // level graph after the iteration in flight
                rc = launch_pdl(ctx, "k_syn_record", k_syn_record, dim3(1), dim3(1), 0, d.syn,
                                (const double*)d.cc, (const unsigned int*)d.max_bits,
                                (const InvState*)d.inv, trace_dev_base, d.trace_cap,
                                ctx->cancel_mapped_dev, h_it, 1);
            }
            cudaGraph_t b2;
            e = cudaStreamEndCapture(ctx->stream, &b2);
            if (!rc && e != cudaSuccess) rc = cuda_fail(e, "iteration capture end");
        }
    }
    ctx->capturing = false;
    ctx->stats.kernel_launches = launches0;
    if (rc) {
        cudaGetLastError();
        return rc;
    }
    const double t1 = tracing() ? now_ms() : 0.0;
    FW_CUDA(cudaGraphInstantiate(&G.e, G.g, 0));
    const double t2 = tracing() ? now_ms() : 0.0;
    // launched without a wait: the next level's pyramid, fields and graph are enqueued behind it
    // while it runs (the executable graph is released when it completes)
    FW_CUDA(cudaGraphLaunch(G.e, ctx->stream));
    ctx->stats.graph_launches++;
    if (tracing())
        std::fprintf(stderr, "[fastwarp] level %d (%lld voxels): capture %.2f ms, instantiate %.2f ms "
                     "(host, overlapping the device)\n", level, (long long)L.grid.count(), t1 - t0,
                     t2 - t1);
    return 0;
}

int check_status(int status, bool masked) {
    if (status > 10) return dense_mi_status(status - 10, masked);
    switch (status) {
        case 0: return 0;
        case 1: return fail(FW_ERR_NOT_FINITE, "syn: the metric gradient is not finite");
        case 2: return fail(FW_ERR_NOT_FINITE, "syn: the displacement field is not finite");
        case 3: return fail(FW_ERR_CANCELLED, "registration cancelled");
        case 4: return fail(FW_ERR_INVALID, std::string("cc metric: ") + FW_NO_VOXEL_IN_MASKS);
        default: return fail(FW_ERR_INVALID, "syn: unknown device status");
    }
}

// Kernels per iteration outside the inversion bodies (for the launch counter).
int kernels_per_iteration(const fw_syn_recipe* r, int mask_warps) {
    int k = r->channels * 3 + (r->channels > 1 ? 2 * r->channels + 2 : 0) +
            4 /*two-pass smoothing or max*/ + 2 /*compose*/ +
            (r->total_field_variance > 0.0 ? 4 : 0) + 1 /*inversion inits*/ + 1 /*record*/ +
            mask_warps + (mask_warps == 2 ? 1 : 0) /*product*/;
    for (int c = 0; c < r->channels; ++c)
        if (r->channel_metrics[c] == FW_METRIC_MATTES) k += 6;  // 7 dense MI kernels, not 1 CC
    return k;
}

__global__ void k_count_nonzero(const float* __restrict__ a, long long n, unsigned int* count) {
    unsigned int c = 0;
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < n;
         l += (long long)gridDim.x * blockDim.x)
        c += a[l] != 0.0f;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// recipe.rs:239-246: a given mask must have a voxel inside.
int check_masks(fw_ctx* ctx, const fw_image* fmask, const fw_image* mmask) {
    const fw_image* ms[2] = {fmask, mmask};
    const char* names[2] = {"fixed", "moving"};
    for (int q = 0; q < 2; ++q) {
        if (!ms[q]) continue;
        unsigned int* cnt = ctx->d_counter + 48;
        FW_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned int), ctx->stream));
        long long n = ms[q]->grid.count();
        unsigned int blocks = (unsigned int)std::min<long long>((n + 255) / 256, 4LL * ctx->num_sms);
        k_count_nonzero<<<std::max(blocks, 1u), 256, 0, ctx->stream>>>(ms[q]->d, n, cnt);
        FW_TRY(check_launch(ctx, "k_count_nonzero"));
        FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, cnt, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                ctx->stream));
        FW_TRY(sync(ctx));
        unsigned int h = 0;
        std::memcpy(&h, ctx->h_pinned, sizeof(h));
        if (h == 0)
            return fail(FW_ERR_INVALID, std::string("syn recipe: the ") + names[q] +
                                            " mask has no voxel inside (every voxel is zero)");
    }
    return 0;
}

}  // namespace

int syn_recipe_check(const fw_syn_recipe* r) { return syn_validate(r); }

int syn_run_device(fw_ctx* ctx, const fw_syn_recipe* r, const fw_image* const* fixed,
                   const fw_image* const* moving, const fw_image* fixed_mask,
                   const fw_image* moving_mask, const fw_affine* initial, const fw_field* prior,
                   const fw_field* prior_inverse, fw_field** warp, fw_field** inverse_warp,
                   fw_syn_iteration* records, int64_t cap, int64_t* count) {
    FW_TRY(syn_validate(r));
    const double t_start = tracing() ? now_ms() : 0.0;
    FW_TRY(check_masks(ctx, fixed_mask, moving_mask));
    const int C = r->channels;
    for (int c = 0; c < C; ++c) FW_CHECK(fixed[c] && moving[c], "syn: null channel image");
    const HostGrid fg = fixed[0]->grid;
    for (int c = 1; c < C; ++c)
        if (!fixed[c]->grid.same(fg)) return fail(FW_ERR_INVALID, "syn: fixed images of the channels differ in grid");
    // syn.rs:803-817: the earlier stages' fields lie on the grid of this stage's last level
    FW_CHECK(!prior == !prior_inverse, "syn: the prior needs both the warp and its inverse");
    if (prior) {
        HostGrid last;
        FW_TRY(level_grid(r, fg, r->levels - 1, last));
        if (!prior->grid.same(last) || !prior_inverse->grid.same(last))
            return fail(FW_ERR_INVALID,
                        "syn: the field of the earlier SyN stages is not on the grid of this "
                        "stage's last level: every SyN stage must end with the same shrink factor");
    }
    int total_iters = 0;
    for (int l = 0; l < r->levels; ++l) total_iters += (int)r->iterations[l];
    // scratch for every reduction of the biggest level, before any capture
    {
        HostGrid last;
        FW_TRY(level_grid(r, fg, r->levels - 1, last));
        FW_TRY(ensure_scratch(ctx, std::max<size_t>(SLOT_PARTIALS + (size_t)(1 << 20),
                                                    inv_scratch_doubles(last))));
    }
    RunScratch rs;
    FW_TRY(rs.init(ctx, C, std::max(total_iters, 1)));
    FW_TRY(upload_syn_dev(ctx, r, rs.d.syn, fixed_mask || moving_mask));
    Level L;
    L.channels = C;
    L.fmask = fixed_mask;
    L.mmask = moving_mask;
    L.prior = prior;
    HostGrid prev;
    bool have_prev = false;
    std::vector<fw_image*> owned;
    auto free_owned = [&]() {
        for (auto* im : owned) fw_image_free(im);
        owned.clear();
    };
    auto free_state = [&]() {
        fw_field* st[] = {L.F, L.Fi, L.M, L.Mi};
        for (auto* f : st) fw_field_free(f);
        L.F = L.Fi = L.M = L.Mi = nullptr;
    };
    int rc = 0;
    int done = 0;
    const bool graphs = use_graphs();
    int graph_levels = 0;
    for (int level = 0; level < r->levels && !rc; ++level) {
        if (cancel_requested(ctx)) {
            rc = fail(FW_ERR_CANCELLED, "registration cancelled");
            break;
        }
        const double t_level = tracing() ? now_ms() : 0.0;
        HostGrid lg;
        rc = level_grid(r, fg, level, lg);
        if (rc) break;
        // level smoothing of the full-resolution images (pyramid.rs:446-460), on the device
        std::vector<const fw_image*> fs(C), ms(C);
        double sigma = r->smoothing_sigmas[level];
        free_owned();
        for (int c = 0; c < C && !rc; ++c) {
            if (sigma > 0.0) {
                double sf[3], sm[3];
                for (int a = 0; a < 3; ++a) {
                    sf[a] = r->sigma_units_mm ? sigma : sigma * fixed[c]->grid.sp[a];
                    sm[a] = r->sigma_units_mm ? sigma : sigma * moving[c]->grid.sp[a];
                }
                fw_image *a = nullptr, *b = nullptr;
                rc = new_image(ctx, fixed[c]->grid, &a);
                if (!rc) owned.push_back(a);
                if (!rc) rc = launch_smooth_recursive(ctx, fixed[c], sf, a);
                if (!rc) rc = new_image(ctx, moving[c]->grid, &b);
                if (!rc) owned.push_back(b);
                if (!rc) rc = launch_smooth_recursive(ctx, moving[c], sm, b);
                fs[c] = a;
                ms[c] = b;
            } else {
                fs[c] = fixed[c];
                ms[c] = moving[c];
            }
        }
        if (rc) break;
        // state fields: zero on the first level, resampled afterwards (syn.rs:850-884)
        fw_field* st[4] = {L.F, L.Fi, L.M, L.Mi};
        fw_field* nx[4] = {nullptr, nullptr, nullptr, nullptr};
        for (int q = 0; q < 4 && !rc; ++q) {
            rc = new_field(ctx, lg, &nx[q]);
            if (rc) break;
            if (!have_prev) {
                FW_CUDA(cudaMemsetAsync(nx[q]->d, 0, nx[q]->bytes, ctx->stream));
            } else if (prev.same(lg)) {
                FW_CUDA(cudaMemcpyAsync(nx[q]->d, st[q]->d, nx[q]->bytes, cudaMemcpyDeviceToDevice, ctx->stream));
            } else {
                rc = launch_resample(ctx, st[q], nx[q]);
            }
        }
        if (rc) {
            for (auto* f : nx) fw_field_free(f);
            break;
        }
        free_state();
        L.F = nx[0];
        L.Fi = nx[1];
        L.M = nx[2];
        L.Mi = nx[3];
        L.grid = lg;
        prev = lg;
        have_prev = true;
        const double t_fields = tracing() ? now_ms() : 0.0;
        free_level_work(L);
        rc = alloc_level_work(ctx, r, L);
        if (rc) break;
        if (tracing())
            std::fprintf(stderr, "[fastwarp] level %d: pyramid and state fields %.2f ms, work buffers "
                         "%.2f ms (host)\n", level, t_fields - t_level, now_ms() - t_fields);
        int limit = (int)r->iterations[level];
        if (limit > 0) {
            if (graphs) {
                // enqueued behind the previous level without waiting for it
                rc = run_level_graph(ctx, r, L, fs, ms, initial, rs.d, level, limit, rs.d.trace);
                if (rc) break;
                ++graph_levels;
                continue;
            }
            rc = run_level_direct(ctx, r, L, fs, ms, initial, rs.d, level, limit, rs.d.trace);
            if (rc) break;
            // the level's status, read after every level (the host drives the loop)
            SynDev h;
            FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, rs.d.syn, sizeof(SynDev), cudaMemcpyDeviceToHost, ctx->stream));
            rc = sync(ctx);
            if (rc) break;
            std::memcpy(&h, ctx->h_pinned, sizeof(h));
            rc = check_status(h.status, fixed_mask || moving_mask);
        }
    }
    // the records of every level and the final status: one read-back after the last level
    if (!rc) {
        SynDev h;
        FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, rs.d.syn, sizeof(SynDev), cudaMemcpyDeviceToHost,
                                ctx->stream));
        rc = sync(ctx);
        if (!rc) {
            std::memcpy(&h, ctx->h_pinned, sizeof(h));
            done = std::min(h.done, std::max(total_iters, 1));
            std::vector<fw_syn_iteration> all((size_t)std::max(done, 1));
            if (done > 0)
                FW_CUDA(cudaMemcpy(all.data(), rs.d.trace, sizeof(fw_syn_iteration) * done,
                                   cudaMemcpyDeviceToHost));
            // the kernels the level graphs ran (direct launches are counted as they are made):
            // every iteration's kernels, three per inversion body, one level init per level
            for (int q = 0; q < done && graphs; ++q) {
                for (int s = 0; s < 4; ++s)
                    ctx->stats.kernel_launches += 3 * (uint64_t)all[q].inversions[s].iterations;
                ctx->stats.kernel_launches +=
                    kernels_per_iteration(r, (fixed_mask ? 1 : 0) + (moving_mask ? 1 : 0));
            }
            if (graphs) ctx->stats.kernel_launches += (uint64_t)graph_levels;
            if (records && cap > 0)
                std::memcpy(records, all.data(),
                            sizeof(fw_syn_iteration) * (size_t)std::min<int64_t>(done, cap));
            rc = check_status(h.status, fixed_mask || moving_mask);
        }
    }
    const double t_end = tracing() ? now_ms() : 0.0;
    free_level_work(L);
    free_owned();
    if (!rc) {
        // syn.rs:969-970: forward = F + Minv(x + F), inverse = M + Finv(x + M)
        fw_field *w = nullptr, *iw = nullptr;
        rc = new_field(ctx, L.grid, &w);
        if (!rc) rc = new_field(ctx, L.grid, &iw);
        if (!rc) rc = launch_compose(ctx, L.Mi, L.F, w, nullptr, 1.0);
        if (!rc) rc = launch_compose(ctx, L.Fi, L.M, iw, nullptr, 1.0);
        if (!rc && prior) {
            // syn.rs:761-774 (collapse): total = W + P(x + W) in place; the inverse needs a
            // new field, total^-1 = Pinv + Winv(x + Pinv)
            fw_field* tiw = nullptr;
            rc = launch_compose(ctx, prior, w, w, nullptr, 1.0);
            if (!rc) rc = new_field(ctx, L.grid, &tiw);
            if (!rc) rc = launch_compose(ctx, iw, prior_inverse, tiw, nullptr, 1.0);
            if (!rc) {
                fw_field_free(iw);
                iw = tiw;
            } else {
                fw_field_free(tiw);
            }
        }
        if (!rc) rc = sync(ctx);
        if (rc) {
            fw_field_free(w);
            fw_field_free(iw);
        } else {
            *warp = w;
            *inverse_warp = iw;
        }
    }
    free_state();
    if (count) *count = done;
    if (tracing())
        std::fprintf(stderr, "[fastwarp] registration: %d iterations, %.2f ms on the host "
                     "(final composition %.2f ms)\n", done, now_ms() - t_start, now_ms() - t_end);
    return rc;
}

}  // namespace fw

using namespace fw;

extern "C" {

int fw_shrink_factors(uint32_t factor, const double spacing[3], uint32_t out[3]) {
    FW_CHECK(spacing && out, "null argument");
    shrink_factors(factor, spacing, out);
    return 0;
}

int fw_shrink_grid(const fw_grid* grid, const uint32_t factors[3], fw_grid* out) {
    FW_CHECK(grid && factors && out, "null argument");
    HostGrid g, o;
    FW_TRY(make_grid(grid, g));
    FW_TRY(shrink_grid(g, factors, o));
    *out = to_c(o);
    return 0;
}

int fw_syn_level_grid(const fw_syn_recipe* recipe, const fw_grid* fixed_grid, int32_t level,
                      fw_grid* out) {
    FW_CHECK(recipe && fixed_grid && out, "null argument");
    FW_TRY(syn_validate(recipe));
    FW_CHECK(level >= 0 && level < recipe->levels, "syn: level out of range");
    HostGrid g, o;
    FW_TRY(make_grid(fixed_grid, g));
    FW_TRY(level_grid(recipe, g, level, o));
    *out = to_c(o);
    return 0;
}

int fw_syn_step(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_image* const* fixed,
                const fw_image* const* moving, const fw_affine* initial, fw_field* f2m,
                fw_field* f2m_inv, fw_field* m2m, fw_field* m2m_inv, double* fixed_update,
                double* moving_update, fw_syn_iteration* record) {
    return fw_syn_step_masked(ctx, recipe, fixed, moving, nullptr, nullptr, initial, f2m, f2m_inv,
                              m2m, m2m_inv, fixed_update, moving_update, record);
}

int fw_syn_step_masked(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_image* const* fixed,
                       const fw_image* const* moving, const fw_image* fixed_mask,
                       const fw_image* moving_mask, const fw_affine* initial, fw_field* f2m,
                       fw_field* f2m_inv, fw_field* m2m, fw_field* m2m_inv, double* fixed_update,
                       double* moving_update, fw_syn_iteration* record) {
    FW_CHECK(ctx && recipe && fixed && moving && f2m && f2m_inv && m2m && m2m_inv, "null argument");
    FW_TRY(syn_validate(recipe));
    FW_TRY(check_masks(ctx, fixed_mask, moving_mask));
    const HostGrid& g = f2m->grid;
    FW_CHECK(f2m_inv->grid.same(g) && m2m->grid.same(g) && m2m_inv->grid.same(g),
             "syn: the state fields differ in grid");
    FW_TRY(ensure_scratch(ctx, std::max<size_t>(SLOT_PARTIALS + (size_t)(1 << 20),
                                                inv_scratch_doubles(g))));
    Level L;
    L.channels = recipe->channels;
    L.fmask = fixed_mask;
    L.mmask = moving_mask;
    L.grid = g;
    L.F = f2m;
    L.Fi = f2m_inv;
    L.M = m2m;
    L.Mi = m2m_inv;
    int rc = alloc_level_work(ctx, recipe, L);
    RunScratch rs;
    if (!rc) rc = rs.init(ctx, L.channels, 1);
    if (!rc) rc = upload_syn_dev(ctx, recipe, rs.d.syn, fixed_mask || moving_mask);
    std::vector<const fw_image*> fs(fixed, fixed + L.channels), ms(moving, moving + L.channels);
    if (!rc) {
        k_syn_level_init<<<1, 1, 0, ctx->stream>>>(rs.d.syn, 0, 1, 0, 0);
        rc = check_launch(ctx, "k_syn_level_init");
    }
    if (!rc) rc = enqueue_iteration(ctx, false, recipe, L, fs, ms, initial, rs.d);
    if (!rc) {
        k_syn_record<<<1, 1, 0, ctx->stream>>>(rs.d.syn, rs.d.cc, rs.d.max_bits, rs.d.inv, rs.d.trace, 1,
                                              nullptr, 0, 0);
        rc = check_launch(ctx, "k_syn_record");
    }
    // the scaled updates of both sides (what the reference passes to compose)
    for (int side = 0; side < 2 && !rc; ++side) {
        double* out = side == 0 ? fixed_update : moving_update;
        if (!out) continue;
        fw_field* u = side == 0 ? (L.sF ? L.sF : (L.accF ? L.accF : L.dF))
                                : (L.sM ? L.sM : (L.accM ? L.accM : L.dM));
        rc = launch_scale_by_max(ctx, u, rs.d.max_bits + side, recipe->gradient_step);
        if (!rc) rc = fw_field_download(ctx, u, out);
    }
    if (!rc) rc = sync(ctx);
    if (!rc && record) {
        FW_CUDA(cudaMemcpy(record, rs.d.trace, sizeof(fw_syn_iteration), cudaMemcpyDeviceToHost));
        record->convergence_value = DBL_MAX;
    }
    if (!rc) {
        SynDev h;
        FW_CUDA(cudaMemcpy(&h, rs.d.syn, sizeof(h), cudaMemcpyDeviceToHost));
        rc = check_status(h.status, fixed_mask || moving_mask);
    }
    L.F = L.Fi = L.M = L.Mi = nullptr;  // owned by the caller
    free_level_work(L);
    return rc;
}

int fw_syn_run_device(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_image* const* fixed,
                      const fw_image* const* moving, const fw_affine* initial,
                      fw_field** warp, fw_field** inverse_warp, fw_syn_iteration* records,
                      int64_t cap, int64_t* count) {
    FW_CHECK(ctx && recipe && fixed && moving && warp && inverse_warp, "null argument");
    return syn_run_device(ctx, recipe, fixed, moving, nullptr, nullptr, initial, nullptr, nullptr,
                          warp, inverse_warp, records, cap, count);
}

int fw_syn_run_device_masked(fw_ctx* ctx, const fw_syn_recipe* recipe,
                             const fw_image* const* fixed, const fw_image* const* moving,
                             const fw_image* fixed_mask, const fw_image* moving_mask,
                             const fw_affine* initial, fw_field** warp, fw_field** inverse_warp,
                             fw_syn_iteration* records, int64_t cap, int64_t* count) {
    FW_CHECK(ctx && recipe && fixed && moving && warp && inverse_warp, "null argument");
    return syn_run_device(ctx, recipe, fixed, moving, fixed_mask, moving_mask, initial, nullptr,
                          nullptr, warp, inverse_warp, records, cap, count);
}

int fw_syn_run_device_from(fw_ctx* ctx, const fw_syn_recipe* recipe,
                           const fw_image* const* fixed, const fw_image* const* moving,
                           const fw_image* fixed_mask, const fw_image* moving_mask,
                           const fw_affine* initial, const fw_field* prior,
                           const fw_field* prior_inverse, fw_field** warp,
                           fw_field** inverse_warp, fw_syn_iteration* records, int64_t cap,
                           int64_t* count) {
    FW_CHECK(ctx && recipe && fixed && moving && warp && inverse_warp, "null argument");
    return syn_run_device(ctx, recipe, fixed, moving, fixed_mask, moving_mask, initial, prior,
                          prior_inverse, warp, inverse_warp, records, cap, count);
}

int fw_syn_run(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_grid* fixed_grid,
               const float* const* fixed, const fw_grid* moving_grid, const float* const* moving,
               const fw_affine* initial, float* warp, float* inverse_warp,
               fw_syn_iteration* records, int64_t cap, int64_t* count) {
    FW_CHECK(ctx && recipe && fixed_grid && fixed && moving_grid && moving && warp && inverse_warp,
             "null argument");
    FW_TRY(syn_validate(recipe));
    const int C = recipe->channels;
    std::vector<fw_image*> fi(C, nullptr), mi(C, nullptr);
    int rc = 0;
    for (int c = 0; c < C && !rc; ++c) {
        rc = fw_image_upload_f32(ctx, fixed_grid, fixed[c], &fi[c]);
        if (!rc) rc = fw_image_upload_f32(ctx, moving_grid, moving[c], &mi[c]);
    }
    fw_field *w = nullptr, *iw = nullptr;
    if (!rc) {
        std::vector<const fw_image*> cf(fi.begin(), fi.end()), cm(mi.begin(), mi.end());
        rc = syn_run_device(ctx, recipe, cf.data(), cm.data(), nullptr, nullptr, initial, nullptr,
                            nullptr, &w, &iw, records, cap, count);
    }
    if (!rc) rc = fw_field_download_f32(ctx, w, warp);
    if (!rc) rc = fw_field_download_f32(ctx, iw, inverse_warp);
    fw_field_free(w);
    fw_field_free(iw);
    for (auto* im : fi) fw_image_free(im);
    for (auto* im : mi) fw_image_free(im);
    return rc;
}

}  // extern "C"
