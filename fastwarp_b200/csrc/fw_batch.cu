// fw_batch.cu -- the batching form: many subjects registered to one template in one SyN run.
//
// The reference registers several moving images against one fixed image only as independent
// runs (register_atlases, crates/fastwarp-cli/src/engine.rs:1016-1072: up to four at a time under
// a split memory budget). Here the subjects of a batch share the template, so every pyramid level
// has ONE level grid for all of them (only the moving sources are ragged: each subject has its
// own grid, affine and smoothed pyramid). Each SyN sub-step (the warps of every channel, the CC
// pairs, the multichannel combination, the smoothing, the compositions and the four inversions)
// is ONE launch over all subjects: a persistent kernel that walks a work list of (subject, tile)
// items. The list lives on the device and is rebuilt by the record kernel at the end of every
// iteration, so a subject that converged (or failed) drops out while the others go on, inside
// the same captured graph. Each level is one CUDA graph: a WHILE node over the iteration, with a
// WHILE node per inversion whose condition is "some subject's inversion runs another body".
//
// Every kernel runs the single-registration kernel's tile body, and every per-subject reduction
// runs in the single kernel's tile order; only the tile shape (z chunk) and the persistent grid
// are the autotuner's choice, so a subject's fields equal its single-registration fields except
// where a reduction grouped by a different tile shape rounds differently in the last bit.
//
// The autotuner (tune_level) times the candidate tile depths and persistent grids of every batched
// kernel family on the level's own buffers, with CUDA events, before the level's graph is
// captured, and keeps the fastest; choices are cached per (level grid, subjects, channels, CC
// radius) for the rest of the process.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "fw_internal.cuh"
#include "fw_syn_state.cuh"

namespace fw {
namespace {

constexpr int BATCH_MAX_SUBJECTS = 256;
constexpr int RECORD_THREADS = 256;

// The work list: active subjects in slot order and their number (BatchList points here).
struct BatchCtl {
    int count;
    int pad[31];
    int active[BATCH_MAX_SUBJECTS];
};

// ---- level start and iteration record of every subject ---------------------------------------

__global__ void __launch_bounds__(RECORD_THREADS) k_batch_level_init(
    SynDev* s, int nsub, int level, int limit, BatchCtl* ctl, cudaGraphConditionalHandle h) {
    __shared__ int run[BATCH_MAX_SUBJECTS];
    for (int b = threadIdx.x; b < nsub; b += blockDim.x) run[b] = syn_level_begin(s + b, level, limit);
    __syncthreads();
    if (threadIdx.x == 0) {
        int n = 0;
        for (int b = 0; b < nsub; ++b)
            if (run[b]) ctl->active[n++] = b;
        ctl->count = n;
        cudaGraphSetConditional(h, n > 0 ? 1u : 0u);
    }
}

// Every active subject's end of iteration (syn_record_step), then the list compacted to the
// subjects whose level goes on (their order kept); the iteration loop runs while any is left.
__global__ void __launch_bounds__(RECORD_THREADS) k_batch_record(
    SynDev* s, const double* __restrict__ cc, int cc_stride, const unsigned int* __restrict__ mx,
    const InvState* __restrict__ inv, fw_syn_iteration* trace, int trace_cap,
    const volatile int* cancel, BatchCtl* ctl, cudaGraphConditionalHandle h) {
    __shared__ int more[BATCH_MAX_SUBJECTS];
    const int n = ctl->count;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int b = ctl->active[i];
        more[i] = syn_record_step(s + b, cc + (size_t)b * cc_stride, mx + 2 * b, inv + 4 * b,
                                  trace + (size_t)b * trace_cap, trace_cap, cancel);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int m = 0;
        for (int i = 0; i < n; ++i)
            if (more[i]) ctl->active[m++] = ctl->active[i];
        ctl->count = m;
        cudaGraphSetConditional(h, m > 0 ? 1u : 0u);
    }
}

// Every subject active (the autotuner's launches).
__global__ void k_batch_all_active(BatchCtl* ctl, int nsub) {
    for (int b = threadIdx.x; b < nsub; b += blockDim.x) ctl->active[b] = b;
    if (threadIdx.x == 0) ctl->count = nsub;
}

// ---- the multichannel combination (syn.rs:218-275) of every active subject ------------------
// grid.y is the subject's slot in the list; the fields are float4 runs of n4 per subject.

// acc += (w / |x|) x when |x| > eps (syn.rs:233-240); on the first channel acc = (w / |x|) x
// (acc = 0 otherwise), the same bits as a cleared accumulator plus the product.
__global__ void k_axpy_norm_batch(float4* __restrict__ acc, const float4* __restrict__ x,
                                  long long n4, long long stride4, const double* __restrict__ nsq,
                                  int nsq_stride, double w, int first, BatchList L) {
    if ((int)blockIdx.y >= *L.count) return;
    const int b = L.active[blockIdx.y];
    const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n4) return;
    float4* ab = acc + b * stride4;
    const double mag = sqrt(nsq[(size_t)b * nsq_stride]);
    if (!(mag > DBL_EPSILON)) {
        if (first) ab[l] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const float a = (float)(w / mag);
    const float4 u = x[b * stride4 + l];
    float4 v = first ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : ab[l];
    v.x = fmaf(a, u.x, v.x);
    v.y = fmaf(a, u.y, v.y);
    v.z = fmaf(a, u.z, v.z);
    v.w = fmaf(a, u.w, v.w);
    ab[l] = v;
}

// acc *= sum_c |d_c| / C (syn.rs:259-263); `which` selects |dF|^2 (1) or |dM|^2 (2).
__global__ void k_scale_norms_batch(float4* __restrict__ acc, long long n4, long long stride4,
                                    const double* __restrict__ cc, int cc_stride, int channels,
                                    int which, BatchList L) {
    if ((int)blockIdx.y >= *L.count) return;
    const int b = L.active[blockIdx.y];
    const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n4) return;
    const double* cb = cc + (size_t)b * cc_stride;
    double tot = 0.0;
    for (int c = 0; c < channels; ++c) tot += sqrt(cb[CC_STRIDE * c + which]);
    const float s = (float)(tot / channels);
    float4 v = acc[b * stride4 + l];
    v.x *= s;
    v.y *= s;
    v.z *= s;
    v.w *= s;
    acc[b * stride4 + l] = v;
}

// ---- tuning ------------------------------------------------------------------------------

struct Tuning {
    int warp_zc = 16, warp_bps = 4;
    int comp_zc = 16, comp_bps = 4;
    int cc_zc = 0, cc_bps = 3;  // cc_zc 0: the whole column
    int step_zc = 1, step_bps = 3;  // inversion step: step tiles per work item, blocks per SM
    int fix_bps = 2;                 // inversion fix kernel
    int smooth_bps = 4;
    double tune_ms = 0.0;
    // the timed best of each batched kernel (one launch over all subjects, ms; body: the whole
    // inversion body, bound + step + fix)
    double warp_ms = 0, cc_ms = 0, smooth_ms = 0, compose_ms = 0, step_ms = 0, body_ms = 0;
    bool cached = false;
};

using TuneKey = std::tuple<int64_t, int64_t, int64_t, int, int, int>;
std::mutex g_tune_mu;
std::map<TuneKey, Tuning> g_tune;

bool tuning_enabled() {
    const char* v = std::getenv("FASTWARP_BATCH_TUNE");
    return !(v && v[0] == '0');
}

// ---- a batch's level -----------------------------------------------------------------------

struct Buf {
    fw_ctx* ctx = nullptr;
    void* p = nullptr;
    size_t bytes = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() { release(); }
    void release() {
        if (p) dev_free(ctx, p, bytes);
        p = nullptr;
        bytes = 0;
    }
    int alloc(fw_ctx* c, size_t b) {
        release();
        ctx = c;
        bytes = b;
        return dev_alloc(c, b, &p);
    }
    float* f() const { return static_cast<float*>(p); }
};

struct BatchLevel {
    HostGrid grid;
    long long n = 0, ps = 0, fs = 0, is = 0;  // voxels, plane stride, field and image strides
    Buf F, Fi, M, Mi;                          // state fields, fs floats per subject
    Buf dF, dM, sF, sM, R, accF, accM;          // work fields
    std::vector<Buf> fmid, mmid;               // warped images per channel, is floats per subject
    std::vector<fw_image*> fixed_s;            // the template's level-smoothed channels (owned)
    std::vector<fw_image*> moving_s;           // [c * B + b] (owned when smoothed)
    bool own_moving = false;
    Buf wargs_f, wargs_m, srcs_f, srcs_m;      // warp arguments and source pointers (device)
    ~BatchLevel() {
        for (auto* im : fixed_s) fw_image_free(im);
        if (own_moving)
            for (auto* im : moving_s) fw_image_free(im);
    }
};

fw_field view(fw_ctx* ctx, const BatchLevel& L, const Buf& b, int s) {
    fw_field f{ctx, L.grid, b.f() + (size_t)s * L.fs, L.ps, (size_t)L.fs * sizeof(float)};
    return f;
}

struct BatchScalars {
    Buf mem;
    SynDev* syn = nullptr;        // [B]
    double* cc = nullptr;         // [B][C * CC_STRIDE]
    unsigned int* mx = nullptr;   // [B][2]
    InvState* inv = nullptr;      // [B][4]
    fw_syn_iteration* trace = nullptr;  // [B][trace_cap]
    BatchCtl* ctl = nullptr;
    unsigned int* counter = nullptr;    // [B]
    int trace_cap = 0, cc_stride = 0;
    int init(fw_ctx* ctx, int B, int C, int cap) {
        auto up = [](size_t x) { return (x + 255) / 256 * 256; };
        trace_cap = std::max(cap, 1);
        cc_stride = C * CC_STRIDE;
        size_t o_syn = 0;
        size_t o_cc = o_syn + up(sizeof(SynDev) * B);
        size_t o_mx = o_cc + up(sizeof(double) * cc_stride * B);
        size_t o_inv = o_mx + up(sizeof(unsigned int) * 2 * B);
        size_t o_ctl = o_inv + up(sizeof(InvState) * 4 * B);
        size_t o_cnt = o_ctl + up(sizeof(BatchCtl));
        size_t o_tr = o_cnt + up(sizeof(unsigned int) * B);
        size_t total = o_tr + sizeof(fw_syn_iteration) * (size_t)trace_cap * B;
        FW_TRY(mem.alloc(ctx, total));
        char* p = static_cast<char*>(mem.p);
        syn = reinterpret_cast<SynDev*>(p + o_syn);
        cc = reinterpret_cast<double*>(p + o_cc);
        mx = reinterpret_cast<unsigned int*>(p + o_mx);
        inv = reinterpret_cast<InvState*>(p + o_inv);
        ctl = reinterpret_cast<BatchCtl*>(p + o_ctl);
        counter = reinterpret_cast<unsigned int*>(p + o_cnt);
        trace = reinterpret_cast<fw_syn_iteration*>(p + o_tr);
        FW_CUDA(cudaMemsetAsync(mem.p, 0, total, ctx->stream));
        return 0;
    }
    BatchList list(int tiles) const { return BatchList{ctl->active, &ctl->count, tiles}; }
};

const fw_invert_params kBatchInvert = {20, 0.001, 0.1, 1};

struct Plan {
    int B, C;
    const fw_syn_recipe* r;
    Tuning t;
    int sms;
    // tiles per subject of each kernel family under the plan's tile shapes
    int warp_tiles(const HostGrid& g) const {
        return (int)(((g.n[0] + 31) / 32) * ((g.n[1] + 7) / 8) * ((g.n[2] + t.warp_zc - 1) / t.warp_zc));
    }
    int comp_tiles(const HostGrid& g) const {
        return (int)(((g.n[0] + 31) / 32) * ((g.n[1] + 7) / 8) * ((g.n[2] + t.comp_zc - 1) / t.comp_zc));
    }
    int cc_zchunk(const HostGrid& g) const { return t.cc_zc > 0 ? t.cc_zc : (int)g.n[2]; }
};

// The autotuner's candidate tile depths: z slices per tile of the gather sweeps (clamped to the
// column), and z slices per CC tile (the column in 1, 2 or 4 chunks, none thinner than the 2r
// filling steps unless the column is).
std::vector<int> gather_zchunks(int nz) {
    std::vector<int> out;
    for (int z : {8, 16, 32, 64}) {
        z = std::min(z, nz);
        if (std::find(out.begin(), out.end(), z) == out.end()) out.push_back(z);
    }
    return out;
}

std::vector<int> cc_zchunks(int nz, int radius) {
    std::vector<int> out;
    for (int k : {1, 2, 4}) {
        const int zc = (nz + k - 1) / k;
        if (k > 1 && zc < 2 * radius) continue;
        if (std::find(out.begin(), out.end(), zc) == out.end()) out.push_back(zc);
    }
    return out;
}

// Partials per subject: the most any batched reduction of the level needs under any candidate
// (and the defaults): 3 doubles per CC tile, 2 per inversion step block (at most one a tile).
long long partials_per_subject(const HostGrid& g, int radius) {
    const int nz = (int)g.n[2];
    long long most = 3LL * cc_batch_tiles(g, nz);
    for (int zc : cc_zchunks(nz, radius)) most = std::max<long long>(most, 3LL * cc_batch_tiles(g, zc));
    most = std::max<long long>(most, 2LL * inv_step_tiles(g));
    return (most + 31) / 32 * 32;
}

struct Run {
    fw_ctx* ctx;
    Plan plan;
    BatchScalars sc;
    Buf partials;
    long long part_stride = 0;
    Buf defer;                  // [B][defer_stride] deferred step warp parts of each subject
    long long defer_stride = 0;
};

// Virtual blocks per subject of the batched fix kernel (its deferred tiles are few).
constexpr int kFixItems = 8;

// The work lists and grids of the level's batched inversion body.
InvBatchBody body_plan(const Run& run, const BatchLevel& L) {
    const Tuning& t = run.plan.t;
    const int sms = run.plan.sms;
    InvBatchBody w;
    w.zchunk = t.step_zc;
    w.bound = run.sc.list(std::min(inv_bound_vblocks(L.grid), 4 * sms));
    w.step = run.sc.list(inv_step_blocks(L.grid, t.step_zc));
    w.fix = run.sc.list(kFixItems);
    w.bound_blocks = 4 * sms;
    w.step_blocks = t.step_bps * sms;
    w.fix_blocks = t.fix_bps * sms;
    return w;
}

int launch_batch_body(Run& run, BatchLevel& L, const InvBatchBody& w, const Buf& field,
                      const Buf& inverse, int q, int which) {
    return launch_inv_body_batch(run.ctx, L.grid, L.ps, w, field.f(), inverse.f(), L.R.f(), L.fs,
                                 (double*)run.partials.p, run.part_stride, run.sc.counter,
                                 run.sc.inv + q, 4, static_cast<unsigned int*>(run.defer.p),
                                 run.defer_stride, which);
}

// The inversion `inverse = invert(field, init inverse)` of every active subject (slot q of the
// four loop states): the loops' settings, then a WHILE node over the body (bound, step, fix).
int enqueue_batch_invert(Run& run, BatchLevel& L, const Buf& field, const Buf& inverse, int q) {
    fw_ctx* ctx = run.ctx;
    const InvBatchBody w = body_plan(run, L);
    cudaStreamCaptureStatus status;
    cudaGraph_t g;
    const cudaGraphNode_t* deps;
    size_t ndeps;
    FW_CUDA(cudaStreamGetCaptureInfo(ctx->stream, &status, nullptr, &g, &deps, &ndeps));
    cudaGraphConditionalHandle h;
    FW_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    FW_TRY(launch_inv_init_batch(ctx, w.step, run.sc.inv + q, 4, kBatchInvert));
    FW_TRY(launch_inv_any(ctx, run.sc.inv + q, 4, w.step, h));
    cudaGraph_t body;
    FW_TRY(add_while_node(ctx->stream, h, &body));
    cudaStream_t main = ctx->stream;
    FW_CUDA(cudaStreamBeginCaptureToGraph(ctx->aux, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
    ctx->stream = ctx->aux;
    int rc = launch_batch_body(run, L, w, field, inverse, q, -1);
    if (!rc) rc = launch_inv_any(ctx, run.sc.inv + q, 4, w.step, h);
    ctx->stream = main;
    cudaGraph_t out;
    cudaError_t e = cudaStreamEndCapture(ctx->aux, &out);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "batched inversion body capture");
    return 0;
}

unsigned int blocks256(long long n) { return (unsigned int)((n + 255) / 256); }

// The kernels of one iteration of every active subject (syn.rs:890-958), in the single driver's
// order, on ctx->stream.
int enqueue_batch_iteration(Run& run, BatchLevel& L) {
    fw_ctx* ctx = run.ctx;
    const Plan& P = run.plan;
    const Tuning& t = P.t;
    const fw_syn_recipe* r = P.r;
    const int C = P.C, B = P.B, sms = P.sms;
    FW_CUDA(cudaMemsetAsync(run.sc.mx, 0, sizeof(unsigned int) * 2 * B, ctx->stream));
    double wsum = 0.0;
    for (int c = 0; c < C; ++c) wsum += r->channel_weights[c];
    const long long n4 = 3 * L.ps / 4, stride4 = L.fs / 4;
    BatchList lw = run.sc.list(P.warp_tiles(L.grid));
    const int cc_zc = P.cc_zchunk(L.grid);
    BatchList lc = run.sc.list(cc_batch_tiles(L.grid, cc_zc));
    BatchList l1 = run.sc.list(1);
    const float* const* srcs_f = static_cast<const float* const*>(L.srcs_f.p);
    const float* const* srcs_m = static_cast<const float* const*>(L.srcs_m.p);
    for (int c = 0; c < C; ++c) {
        // the template through F^-1 (shared arguments), each subject's source through its affine
        // and M^-1
        FW_TRY(launch_warp_batch(ctx, L.wargs_f.p, srcs_f + c, 0, L.grid, t.warp_zc, lw,
                                 t.warp_bps * sms, L.Fi.f(), L.fs, L.fmid[c].f(), L.is));
        FW_TRY(launch_warp_batch(ctx, L.wargs_m.p, srcs_m + (size_t)c * B, 1, L.grid, t.warp_zc,
                                 lw, t.warp_bps * sms, L.Mi.f(), L.fs, L.mmid[c].f(), L.is));
        FW_TRY(launch_cc_pair_batch(ctx, L.grid, L.ps, r->cc_radius, cc_zc, lc, t.cc_bps * sms,
                                    L.fmid[c].f(), L.mmid[c].f(), L.is, L.dF.f(), L.dM.f(), L.fs,
                                    (double*)run.partials.p, run.part_stride, run.sc.counter,
                                    run.sc.cc + CC_STRIDE * c, run.sc.cc_stride, C > 1 ? 1 : 0));
        if (C > 1) {
            const double wn = r->channel_weights[c] / wsum;
            const dim3 g(blocks256(n4), B);
            k_axpy_norm_batch<<<g, 256, 0, ctx->stream>>>((float4*)L.accF.p, (const float4*)L.dF.p,
                                                         n4, stride4, run.sc.cc + CC_STRIDE * c + 1,
                                                         run.sc.cc_stride, wn, c == 0, l1);
            FW_TRY(check_launch(ctx, "k_axpy_norm_batch"));
            k_axpy_norm_batch<<<g, 256, 0, ctx->stream>>>((float4*)L.accM.p, (const float4*)L.dM.p,
                                                         n4, stride4, run.sc.cc + CC_STRIDE * c + 2,
                                                         run.sc.cc_stride, wn, c == 0, l1);
            FW_TRY(check_launch(ctx, "k_axpy_norm_batch"));
        }
    }
    const Buf* gF = &L.dF;
    const Buf* gM = &L.dM;
    if (C > 1) {
        const dim3 g(blocks256(n4), B);
        k_scale_norms_batch<<<g, 256, 0, ctx->stream>>>((float4*)L.accF.p, n4, stride4, run.sc.cc,
                                                       run.sc.cc_stride, C, 1, l1);
        FW_TRY(check_launch(ctx, "k_scale_norms_batch"));
        k_scale_norms_batch<<<g, 256, 0, ctx->stream>>>((float4*)L.accM.p, n4, stride4, run.sc.cc,
                                                       run.sc.cc_stride, C, 2, l1);
        FW_TRY(check_launch(ctx, "k_scale_norms_batch"));
        gF = &L.accF;
        gM = &L.accM;
    }
    // update_total_field of both sides (syn.rs:422-445), one side after the other
    struct Side {
        const Buf* g;
        Buf* s;
        Buf* field;
        Buf* inverse;
        int side;
    } sides[2] = {{gF, &L.sF, &L.F, &L.Fi, 0}, {gM, &L.sM, &L.M, &L.Mi, 1}};
    BatchList lcomp = run.sc.list(P.comp_tiles(L.grid));
    for (auto& s : sides) {
        FW_TRY(launch_smooth_batch(ctx, L.grid, L.ps, r->update_field_variance, run.sc.ctl->active,
                                   &run.sc.ctl->count, t.smooth_bps * sms, t.smooth_bps * sms,
                                   s.g->f(), s.s->f(), L.R.f(), L.fs, run.sc.mx + s.side, 2));
        FW_TRY(launch_compose_batch(ctx, L.grid, L.ps, t.comp_zc, lcomp, t.comp_bps * sms,
                                    s.s->f(), s.field->f(), L.fs, run.sc.mx + s.side, 2,
                                    r->gradient_step));
        FW_TRY(enqueue_batch_invert(run, L, *s.field, *s.inverse, 2 * s.side));
        FW_TRY(enqueue_batch_invert(run, L, *s.inverse, *s.field, 2 * s.side + 1));
    }
    return 0;
}

// ---- the autotuner ---------------------------------------------------------------------------

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

// Mean ms of `reps` launches by `launch` after one warm-up (CUDA events on the stream).
template <typename F>
int time_launch(fw_ctx* ctx, Timer& tm, int reps, F launch, double* ms) {
    FW_TRY(launch());
    FW_CUDA(cudaEventRecord(tm.a, ctx->stream));
    for (int i = 0; i < reps; ++i) FW_TRY(launch());
    FW_CUDA(cudaEventRecord(tm.b, ctx->stream));
    FW_CUDA(cudaEventSynchronize(tm.b));
    float t = 0.0f;
    FW_CUDA(cudaEventElapsedTime(&t, tm.a, tm.b));
    *ms = (double)t / reps;
    return 0;
}

// Picks the tile depths and persistent grids of the level's batched kernels by timing them on
// the level's buffers (every subject active); the state fields are only read. Scratch use: the
// warped images, dF/dM/sF/sM/R and the loop states, all rewritten by the iteration.
int tune_level(Run& run, BatchLevel& L, Tuning& best) {
    fw_ctx* ctx = run.ctx;
    const Plan& P = run.plan;
    const int B = P.B, sms = P.sms, reps = 2;
    Timer tm;
    k_batch_all_active<<<1, 256, 0, ctx->stream>>>(run.sc.ctl, B);
    FW_TRY(check_launch(ctx, "k_batch_all_active"));
    const float* const* srcs_m = static_cast<const float* const*>(L.srcs_m.p);
    const float* const* srcs_f = static_cast<const float* const*>(L.srcs_f.p);
    const int nz = (int)L.grid.n[2];
    const std::vector<int> gz = gather_zchunks(nz);
    double ms = 0.0, bestms;
    // the moving-side warp (the gather through each subject's own source)
    bestms = DBL_MAX;
    for (int zc : gz) {
        const int tiles = (int)(((L.grid.n[0] + 31) / 32) * ((L.grid.n[1] + 7) / 8) * ((nz + zc - 1) / zc));
        FW_TRY(time_launch(ctx, tm, reps, [&] {
            return launch_warp_batch(ctx, L.wargs_m.p, srcs_m, 1, L.grid, zc, run.sc.list(tiles),
                                     best.warp_bps * sms, L.Mi.f(), L.fs, L.mmid[0].f(), L.is);
        }, &ms));
        if (ms < bestms) bestms = ms, best.warp_zc = zc;
    }
    bestms = DBL_MAX;
    for (int bps : {2, 4, 8}) {
        const int zc = best.warp_zc;
        const int tiles = (int)(((L.grid.n[0] + 31) / 32) * ((L.grid.n[1] + 7) / 8) * ((nz + zc - 1) / zc));
        FW_TRY(time_launch(ctx, tm, reps, [&] {
            return launch_warp_batch(ctx, L.wargs_m.p, srcs_m, 1, L.grid, zc, run.sc.list(tiles),
                                     bps * sms, L.Mi.f(), L.fs, L.mmid[0].f(), L.is);
        }, &ms));
        if (ms < bestms) bestms = ms, best.warp_bps = bps;
    }
    best.warp_ms = bestms;
    // the CC pair on the warped template and subject: z chunks per column (whole columns pay
    // the 2r filling steps once)
    {
        const int zc = best.warp_zc;
        const int tiles = (int)(((L.grid.n[0] + 31) / 32) * ((L.grid.n[1] + 7) / 8) * ((nz + zc - 1) / zc));
        FW_TRY(launch_warp_batch(ctx, L.wargs_f.p, srcs_f, 0, L.grid, zc, run.sc.list(tiles),
                                 best.warp_bps * sms, L.Fi.f(), L.fs, L.fmid[0].f(), L.is));
    }
    const int R = P.r->cc_radius;
    const int occ = std::max(1, cc_batch_blocks_per_sm(R));
    bestms = DBL_MAX;
    for (int zc : cc_zchunks(nz, R)) {
        FW_TRY(time_launch(ctx, tm, reps, [&] {
            return launch_cc_pair_batch(ctx, L.grid, L.ps, R, zc, run.sc.list(cc_batch_tiles(L.grid, zc)),
                                        occ * sms, L.fmid[0].f(), L.mmid[0].f(), L.is, L.dF.f(),
                                        L.dM.f(), L.fs, (double*)run.partials.p, run.part_stride,
                                        run.sc.counter, run.sc.cc, run.sc.cc_stride, 1);
        }, &ms));
        if (ms < bestms) bestms = ms, best.cc_zc = zc == nz ? 0 : zc;
    }
    best.cc_bps = occ;
    best.cc_ms = bestms;
    // the smoothing pair (into sF, with R as its temporary)
    bestms = DBL_MAX;
    for (int bps : {2, 4, 8}) {
        FW_TRY(time_launch(ctx, tm, reps, [&] {
            return launch_smooth_batch(ctx, L.grid, L.ps, P.r->update_field_variance,
                                       run.sc.ctl->active, &run.sc.ctl->count, bps * sms,
                                       bps * sms, L.dF.f(), L.sF.f(), L.R.f(), L.fs, run.sc.mx, 2);
        }, &ms));
        if (ms < bestms) bestms = ms, best.smooth_bps = bps;
    }
    best.smooth_ms = bestms;
    // the composition, in place on a scratch copy (dM) of the level's field F with sF as the
    // update: the gathers land where the iteration's will
    FW_CUDA(cudaMemcpyAsync(L.dM.p, L.F.p, L.dM.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    bestms = DBL_MAX;
    for (int zc : gz) {
        for (int bps : {2, 4, 8}) {
            const int tiles = (int)(((L.grid.n[0] + 31) / 32) * ((L.grid.n[1] + 7) / 8) * ((nz + zc - 1) / zc));
            FW_TRY(time_launch(ctx, tm, reps, [&] {
                return launch_compose_batch(ctx, L.grid, L.ps, zc, run.sc.list(tiles), bps * sms,
                                            L.sF.f(), L.dM.f(), L.fs, run.sc.mx, 2, 1e-6);
            }, &ms));
            if (ms < bestms) bestms = ms, best.comp_zc = zc, best.comp_bps = bps;
        }
    }
    best.compose_ms = bestms;
    // the inversion step (with its bound) of F^-1 against F on a scratch copy (dM) of the level's
    // inverse, loop states of slot 0 kept iterating; then the whole body with the best grid
    FW_CUDA(cudaMemcpyAsync(L.dM.p, L.Fi.p, L.dM.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    const fw_invert_params forever = {1 << 30, -1.0, -1.0, 1};
    FW_TRY(launch_inv_init_batch(ctx, run.sc.list(1), run.sc.inv, 4, forever));
    bestms = DBL_MAX;
    // step tiles per work item: as the single step plans them, or twice as many (fewer items and
    // partials per subject; the subject's mean is then summed in other groups, a last-bit change)
    const int zc1 = inv_step_zchunk(L.grid.n, sms);
    const long long gzs =  // step tiles along z
        inv_step_tiles(L.grid) / (((L.grid.n[0] + 31) / 32) * ((L.grid.n[1] + 7) / 8));
    for (int zc : {zc1, 2 * zc1}) {
        if (zc != zc1 && zc > gzs) continue;
        for (int bps : {2, 3, 4}) {
            run.plan.t.step_zc = zc;
            run.plan.t.step_bps = bps;
            const InvBatchBody w = body_plan(run, L);
            // every step after its own bound (which also clears the deferred lists)
            FW_TRY(time_launch(ctx, tm, reps, [&] {
                FW_TRY(launch_batch_body(run, L, w, L.F, L.dM, 0, 0));
                return launch_batch_body(run, L, w, L.F, L.dM, 0, 1);
            }, &ms));
            if (ms < bestms) bestms = ms, best.step_bps = bps, best.step_zc = zc;
        }
    }
    best.step_ms = bestms;
    run.plan.t.step_zc = best.step_zc;
    run.plan.t.step_bps = best.step_bps;
    {
        const InvBatchBody w = body_plan(run, L);
        FW_TRY(time_launch(ctx, tm, reps, [&] {
            return launch_batch_body(run, L, w, L.F, L.dM, 0, -1);
        }, &ms));
        best.body_ms = ms;
    }
    FW_CUDA(cudaMemsetAsync(run.sc.inv, 0, sizeof(InvState) * 4 * B, ctx->stream));
    FW_CUDA(cudaMemsetAsync(run.sc.mx, 0, sizeof(unsigned int) * 2 * B, ctx->stream));
    return sync(ctx);
}

// ---- levels ----------------------------------------------------------------------------------

int level_grid_of(const fw_syn_recipe* r, const HostGrid& fg, int level, HostGrid& out) {
    const fw_grid c = to_c(fg);
    fw_grid lg;
    FW_TRY(fw_syn_level_grid(r, &c, level, &lg));
    return make_grid(&lg, out);
}

// Allocates the level's buffers and fills the state fields: zero on the first level, else each
// subject's previous state resampled onto the new grid (syn.rs:850-884).
int setup_level(Run& run, BatchLevel& L, const BatchLevel* prev, const HostGrid& lg) {
    fw_ctx* ctx = run.ctx;
    const int B = run.plan.B, C = run.plan.C;
    L.grid = lg;
    L.n = lg.count();
    L.ps = plane_stride(L.n);
    L.fs = 3 * L.ps;
    L.is = plane_stride(L.n);
    const size_t fb = sizeof(float) * (size_t)L.fs * B, ib = sizeof(float) * (size_t)L.is * B;
    Buf* state[4] = {&L.F, &L.Fi, &L.M, &L.Mi};
    for (Buf* b : state) FW_TRY(b->alloc(ctx, fb));
    if (!prev) {
        for (Buf* b : state) FW_CUDA(cudaMemsetAsync(b->p, 0, fb, ctx->stream));
    } else {
        const Buf* old[4] = {&prev->F, &prev->Fi, &prev->M, &prev->Mi};
        for (int q = 0; q < 4; ++q)
            for (int s = 0; s < B; ++s) {
                fw_field src = view(ctx, *prev, *old[q], s);
                fw_field dst = view(ctx, L, *state[q], s);
                if (prev->grid.same(lg))
                    FW_CUDA(cudaMemcpyAsync(dst.d, src.d, dst.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
                else
                    FW_TRY(launch_resample(ctx, &src, &dst));
            }
    }
    Buf* work[5] = {&L.dF, &L.dM, &L.sF, &L.sM, &L.R};
    for (Buf* b : work) FW_TRY(b->alloc(ctx, fb));
    if (C > 1) {
        FW_TRY(L.accF.alloc(ctx, fb));
        FW_TRY(L.accM.alloc(ctx, fb));
    }
    L.fmid = std::vector<Buf>(C);
    L.mmid = std::vector<Buf>(C);
    for (int c = 0; c < C; ++c) {
        FW_TRY(L.fmid[c].alloc(ctx, ib));
        FW_TRY(L.mmid[c].alloc(ctx, ib));
    }
    return 0;
}

// The level's smoothed images (pyramid.rs:446-460) and the warp arguments on the device.
int setup_sources(Run& run, BatchLevel& L, const fw_image* const* fixed,
                  const fw_batch_subject* subj, const HostGrid& fg, double sigma) {
    fw_ctx* ctx = run.ctx;
    const fw_syn_recipe* r = run.plan.r;
    const int B = run.plan.B, C = run.plan.C;
    std::vector<const float*> sf(C), sm((size_t)C * B);
    L.own_moving = sigma > 0.0;
    for (int c = 0; c < C; ++c) {
        const fw_image* f = fixed[c];
        if (sigma > 0.0) {
            double s3[3];
            for (int a = 0; a < 3; ++a) s3[a] = r->sigma_units_mm ? sigma : sigma * f->grid.sp[a];
            fw_image* im = nullptr;
            FW_TRY(new_image(ctx, f->grid, &im));
            L.fixed_s.push_back(im);
            FW_TRY(launch_smooth_recursive(ctx, f, s3, im));
            f = im;
        }
        sf[c] = f->d;
        for (int b = 0; b < B; ++b) {
            const fw_image* m = subj[b].moving[c];
            if (sigma > 0.0) {
                double s3[3];
                for (int a = 0; a < 3; ++a) s3[a] = r->sigma_units_mm ? sigma : sigma * m->grid.sp[a];
                fw_image* im = nullptr;
                FW_TRY(new_image(ctx, m->grid, &im));
                L.moving_s.push_back(im);
                FW_TRY(launch_smooth_recursive(ctx, m, s3, im));
                m = im;
            }
            sm[(size_t)c * B + b] = m->d;
        }
    }
    const size_t wa = warp_args_size();
    std::vector<unsigned char> hf(wa), hm(wa * B);
    fill_warp_args(fg, L.grid, L.ps, nullptr, hf.data());
    for (int b = 0; b < B; ++b)
        fill_warp_args(subj[b].moving[0]->grid, L.grid, L.ps,
                       subj[b].has_initial ? &subj[b].initial : nullptr, hm.data() + wa * b);
    FW_TRY(L.wargs_f.alloc(ctx, wa));
    FW_TRY(L.wargs_m.alloc(ctx, wa * B));
    FW_TRY(L.srcs_f.alloc(ctx, sizeof(float*) * C));
    FW_TRY(L.srcs_m.alloc(ctx, sizeof(float*) * C * B));
    FW_CUDA(cudaMemcpyAsync(L.wargs_f.p, hf.data(), wa, cudaMemcpyHostToDevice, ctx->stream));
    FW_CUDA(cudaMemcpyAsync(L.wargs_m.p, hm.data(), wa * B, cudaMemcpyHostToDevice, ctx->stream));
    FW_CUDA(cudaMemcpyAsync(L.srcs_f.p, sf.data(), sizeof(float*) * C, cudaMemcpyHostToDevice,
                            ctx->stream));
    FW_CUDA(cudaMemcpyAsync(L.srcs_m.p, sm.data(), sizeof(float*) * C * B, cudaMemcpyHostToDevice,
                            ctx->stream));
    return sync(ctx);  // the host staging above lives on this stack frame
}

struct GraphGuard {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~GraphGuard() {
        if (e) cudaGraphExecDestroy(e);
        if (g) cudaGraphDestroy(g);
    }
};

// Captures the level's iteration loop of every subject as one graph, launches it and waits;
// the device time of the launch goes to *ms.
int run_level(Run& run, BatchLevel& L, int level, int limit, double* ms) {
    fw_ctx* ctx = run.ctx;
    GraphGuard G;
    FW_CUDA(cudaGraphCreate(&G.g, 0));
    cudaGraphConditionalHandle h_it = 0;
    FW_CUDA(cudaGraphConditionalHandleCreate(&h_it, G.g, 0, 0));
    FW_CUDA(cudaStreamBeginCaptureToGraph(ctx->stream, G.g, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
    ctx->capturing = true;
    const uint64_t launches0 = ctx->stats.kernel_launches;
    int rc = 0;
    cudaGraph_t body = nullptr;
    k_batch_level_init<<<1, RECORD_THREADS, 0, ctx->stream>>>(run.sc.syn, run.plan.B, level, limit,
                                                              run.sc.ctl, h_it);
    rc = check_launch(ctx, "k_batch_level_init");
    if (!rc) rc = add_while_node(ctx->stream, h_it, &body);
    cudaGraph_t top;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &top);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "batch level capture");
    if (!rc) {
        e = cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed);
        if (e != cudaSuccess) rc = cuda_fail(e, "batch iteration capture");
        if (!rc) {
            rc = enqueue_batch_iteration(run, L);
            if (!rc) {
                k_batch_record<<<1, RECORD_THREADS, 0, ctx->stream>>>(
                    run.sc.syn, run.sc.cc, run.sc.cc_stride, run.sc.mx, run.sc.inv,
                    run.sc.trace, run.sc.trace_cap, ctx->cancel_mapped_dev, run.sc.ctl, h_it);
                rc = check_launch(ctx, "k_batch_record");
            }
            cudaGraph_t b2;
            e = cudaStreamEndCapture(ctx->stream, &b2);
            if (!rc && e != cudaSuccess) rc = cuda_fail(e, "batch iteration capture end");
        }
    }
    ctx->capturing = false;
    ctx->stats.kernel_launches = launches0;
    if (rc) {
        cudaGetLastError();
        return rc;
    }
    FW_CUDA(cudaGraphInstantiate(&G.e, G.g, 0));
    Timer tm;
    FW_CUDA(cudaEventRecord(tm.a, ctx->stream));
    FW_CUDA(cudaGraphLaunch(G.e, ctx->stream));
    FW_CUDA(cudaEventRecord(tm.b, ctx->stream));
    ctx->stats.graph_launches++;
    FW_TRY(sync(ctx));
    float t = 0.0f;
    FW_CUDA(cudaEventElapsedTime(&t, tm.a, tm.b));
    *ms = t;
    return 0;
}

int upload_syn_devs(fw_ctx* ctx, const fw_syn_recipe* r, SynDev* d, int B) {
    std::vector<SynDev> h((size_t)B);
    for (auto& x : h) {
        std::memset(&x, 0, sizeof(x));
        for (int c = 0; c < r->channels; ++c) x.metric[c] = r->channel_metrics[c];
        x.window = r->convergence_window;
        x.threshold = r->convergence_threshold;
        x.step = r->gradient_step;
        x.channels = r->channels;
        double ws = 0.0;
        for (int c = 0; c < r->channels; ++c) ws += r->channel_weights[c];
        for (int c = 0; c < r->channels; ++c) x.wnorm[c] = r->channel_weights[c] / ws;
    }
    FW_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(SynDev) * B, cudaMemcpyHostToDevice, ctx->stream));
    return sync(ctx);
}

int subject_status(int status) {
    switch (status) {
        case 0: return FW_OK;
        case 3: return FW_ERR_CANCELLED;
        case 1:
        case 2: return FW_ERR_NOT_FINITE;
        default: return FW_ERR_INVALID;
    }
}

}  // namespace

int batch_syn_run(fw_ctx* ctx, const fw_syn_recipe* r, const fw_image* const* fixed, int nsub,
                  const fw_batch_subject* subj, fw_field** warps, fw_field** inverses,
                  fw_syn_iteration* records, int64_t cap, int64_t* counts, int32_t* statuses,
                  fw_batch_report* report) {
    FW_CHECK(nsub >= 1 && nsub <= BATCH_MAX_SUBJECTS, "batched SyN: 1..=256 subjects");
    const int C = r->channels, B = nsub;
    for (int c = 0; c < C; ++c) {
        FW_CHECK(r->channel_metrics[c] == FW_METRIC_CC, "batched SyN: CC channels only");
        FW_CHECK(fixed[c], "batched SyN: null template channel");
        FW_CHECK(fixed[c]->grid.same(fixed[0]->grid),
                 "batched SyN: the template's channels differ in grid");
    }
    FW_CHECK(r->update_field_variance > 0.0,
             "batched SyN: the update field must be smoothed (variance > 0)");
    FW_CHECK(!(r->total_field_variance > 0.0),
             "batched SyN: total-field smoothing is not supported in a batch");
    for (int b = 0; b < B; ++b)
        for (int c = 0; c < C; ++c) {
            FW_CHECK(subj[b].moving[c], "batched SyN: null subject image");
            FW_CHECK(subj[b].moving[c]->grid.same(subj[b].moving[0]->grid),
                     "batched SyN: a subject's channels differ in grid");
        }
    const HostGrid fg = fixed[0]->grid;
    int total_iters = 0;
    for (int l = 0; l < r->levels; ++l) total_iters += (int)r->iterations[l];
    Run run;
    run.ctx = ctx;
    run.plan.B = B;
    run.plan.C = C;
    run.plan.r = r;
    run.plan.sms = ctx->num_sms;
    FW_TRY(run.sc.init(ctx, B, C, std::max(total_iters, 1)));
    FW_TRY(upload_syn_devs(ctx, r, run.sc.syn, B));
    if (report) {
        std::memset(report, 0, sizeof(*report));
        report->subjects = B;
        report->levels = r->levels;
    }
    const uint64_t live0 = ctx->live_bytes.load();
    uint64_t peak = 0;
    std::unique_ptr<BatchLevel> prev, cur;
    for (int level = 0; level < r->levels; ++level) {
        if (cancel_requested(ctx)) return fail(FW_ERR_CANCELLED, "registration cancelled");
        const auto t_level = std::chrono::steady_clock::now();
        HostGrid lg;
        FW_TRY(level_grid_of(r, fg, level, lg));
        cur.reset(new BatchLevel());
        FW_TRY(setup_level(run, *cur, prev.get(), lg));
        prev.reset();  // the previous level's buffers go back to the cache
        FW_TRY(setup_sources(run, *cur, fixed, subj, fg, r->smoothing_sigmas[level]));
        const long long pps = partials_per_subject(lg, r->cc_radius);
        if (pps > run.part_stride) {
            run.part_stride = pps;
            FW_TRY(run.partials.alloc(ctx, sizeof(double) * (size_t)pps * B));
        }
        const long long dps = (inv_step_parts(lg) + 63) / 64 * 64;
        if (dps > run.defer_stride) {
            run.defer_stride = dps;
            FW_TRY(run.defer.alloc(ctx, sizeof(unsigned int) * (size_t)dps * B));
        }
        if (report) {
            FW_TRY(sync(ctx));
            report->prepare_ms[level] =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_level).count();
        }
        // the tile shapes and grids of this level: cached, tuned, or the defaults
        Tuning t;
        const TuneKey key{lg.n[0], lg.n[1], lg.n[2], B, C, r->cc_radius};
        bool have = false;
        {
            std::lock_guard<std::mutex> lock(g_tune_mu);
            auto it = g_tune.find(key);
            if (it != g_tune.end()) {
                t = it->second;
                t.cached = true;
                have = true;
            }
        }
        if (!have && tuning_enabled()) {
            const auto t0 = std::chrono::steady_clock::now();
            run.plan.t = t;
            FW_TRY(tune_level(run, *cur, t));
            t.tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            std::lock_guard<std::mutex> lock(g_tune_mu);
            g_tune[key] = t;
        }
        if (!t.cached && !tuning_enabled()) t.step_zc = inv_step_zchunk(lg.n, ctx->num_sms);
        run.plan.t = t;
        peak = std::max<uint64_t>(peak, ctx->live_bytes.load() - live0);
        double ms = 0.0;
        const int limit = (int)r->iterations[level];
        if (limit > 0) FW_TRY(run_level(run, *cur, level, limit, &ms));
        if (report) {
            fw_batch_tuning& o = report->tuning[level];
            o.level = level;
            for (int a = 0; a < 3; ++a) o.grid_size[a] = lg.n[a];
            o.warp_zchunk = t.warp_zc;
            o.warp_blocks_per_sm = t.warp_bps;
            o.compose_zchunk = t.comp_zc;
            o.compose_blocks_per_sm = t.comp_bps;
            o.cc_zchunk = t.cc_zc > 0 ? t.cc_zc : (int)lg.n[2];
            o.cc_blocks_per_sm = t.cc_bps;
            o.measure_zchunk = t.step_zc;
            o.measure_blocks_per_sm = t.step_bps;
            o.body_blocks_per_sm = t.fix_bps;
            o.smooth_blocks_per_sm = t.smooth_bps;
            o.from_cache = t.cached ? 1 : 0;
            o.tune_ms = t.tune_ms;
            o.kernel_ms[0] = t.warp_ms;
            o.kernel_ms[1] = t.cc_ms;
            o.kernel_ms[2] = t.smooth_ms;
            o.kernel_ms[3] = t.compose_ms;
            o.kernel_ms[4] = t.step_ms;
            o.kernel_ms[5] = t.body_ms;
            report->level_ms[level] = ms;
        }
        // the smoothed sources of this level are not needed by the next one
        for (auto* im : cur->fixed_s) fw_image_free(im);
        cur->fixed_s.clear();
        if (cur->own_moving)
            for (auto* im : cur->moving_s) fw_image_free(im);
        cur->moving_s.clear();
        prev = std::move(cur);
    }
    // every subject's status, records and final fields (syn.rs:969-970)
    const auto t_finish = std::chrono::steady_clock::now();
    std::vector<SynDev> h((size_t)B);
    FW_CUDA(cudaMemcpyAsync(h.data(), run.sc.syn, sizeof(SynDev) * B, cudaMemcpyDeviceToHost,
                            ctx->stream));
    FW_TRY(sync(ctx));
    const BatchLevel& L = *prev;
    for (int b = 0; b < B; ++b) {
        const int done = std::min(h[b].done, std::max(total_iters, 1));
        if (counts) counts[b] = done;
        if (records && cap > 0 && done > 0)
            FW_CUDA(cudaMemcpy(records + (size_t)b * cap, run.sc.trace + (size_t)b * run.sc.trace_cap,
                               sizeof(fw_syn_iteration) * (size_t)std::min<int64_t>(done, cap),
                               cudaMemcpyDeviceToHost));
        const int st = subject_status(h[b].status);
        if (statuses) statuses[b] = st;
        warps[b] = inverses[b] = nullptr;
        if (st != FW_OK) continue;
        fw_field F = view(ctx, L, L.F, b), Fi = view(ctx, L, L.Fi, b);
        fw_field M = view(ctx, L, L.M, b), Mi = view(ctx, L, L.Mi, b);
        fw_field *w = nullptr, *iw = nullptr;
        int rc = new_field(ctx, L.grid, &w);
        if (!rc) rc = new_field(ctx, L.grid, &iw);
        if (!rc) rc = launch_compose(ctx, &Mi, &F, w, nullptr, 1.0);
        if (!rc) rc = launch_compose(ctx, &Fi, &M, iw, nullptr, 1.0);
        if (rc) {
            fw_field_free(w);
            fw_field_free(iw);
            for (int q = 0; q < b; ++q) {
                fw_field_free(warps[q]);
                fw_field_free(inverses[q]);
                warps[q] = inverses[q] = nullptr;
            }
            return rc;
        }
        warps[b] = w;
        inverses[b] = iw;
    }
    if (report) report->device_bytes = peak;
    FW_TRY(sync(ctx));
    if (report)
        report->finish_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_finish).count();
    return 0;
}

}  // namespace fw

using namespace fw;

extern "C" int fw_batch_syn_run(fw_ctx* ctx, const fw_syn_recipe* recipe,
                                const fw_image* const* fixed, int32_t subjects,
                                const fw_batch_subject* subject, fw_field** warps,
                                fw_field** inverse_warps, fw_syn_iteration* records, int64_t cap,
                                int64_t* counts, int32_t* statuses, fw_batch_report* report) {
    FW_CHECK(ctx && recipe && fixed && subject && warps && inverse_warps, "null argument");
    FW_TRY(syn_recipe_check(recipe));
    return batch_syn_run(ctx, recipe, fixed, subjects, subject, warps, inverse_warps, records,
                         cap, counts, statuses, report);
}
