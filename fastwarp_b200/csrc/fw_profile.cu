// fw_profile.cu -- per-kernel device timing with CUDA events on the context's stream (the
// timestamp profiler of the wgpu engine, crates/fastwarp-gpu/src/profiler.rs:8-60, for the
// kernels of one SyN iteration at a given level grid).
#include <cuda_runtime.h>

#include <cstring>

#include "fw_internal.cuh"

namespace fw {
namespace {

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    ~Events() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

}  // namespace
}  // namespace fw

using namespace fw;

extern "C" {

/* Times `reps` back-to-back launches of each kernel of a SyN iteration on the grid of `fixed`
 * (fixed and moving on one grid) and writes the mean milliseconds per launch and the
 * algorithmic bytes per launch:
 *   [0] warp (field + source gather + output), [1] CC pair (2 images in, 2 fields out),
 *   [2] Gaussian smoothing with the max norm, [3] compose+scale in place,
 *   [4] one inversion body as the loop runs it (its bound, step and fix kernels, after the loop's
 *   init), [5] the bound kernel alone, [6] the fix kernel alone (the tiles the step deferred;
 *   bytes counts their voxels). */
int fw_time_kernels(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving, int32_t radius,
                    double variance, int32_t reps, double ms[7], double bytes[7]) {
    FW_CHECK(ctx && fixed && moving && ms && bytes && reps > 0, "null argument");
    FW_CHECK(fixed->grid.same(moving->grid), "time kernels: the images are not on one grid");
    const HostGrid& g = fixed->grid;
    const double n = (double)g.count();
    fw_field *u = nullptr, *a = nullptr, *b = nullptr, *s = nullptr, *w = nullptr, *e = nullptr;
    fw_image* out = nullptr;
    fw_grid cg = to_c(g);
    int rc = fw_field_zero(ctx, &cg, &u);
    if (!rc) rc = fw_field_zero(ctx, &cg, &a);
    if (!rc) rc = fw_field_zero(ctx, &cg, &b);
    if (!rc) rc = fw_field_zero(ctx, &cg, &s);
    if (!rc) rc = fw_field_zero(ctx, &cg, &w);
    if (!rc) rc = fw_field_zero(ctx, &cg, &e);
    if (!rc) rc = new_image(ctx, g, &out);
    if (!rc) rc = ensure_scratch(ctx, SLOT_PARTIALS + (size_t)(1 << 20));
    Events ev;
    if (!rc && (cudaEventCreate(&ev.a) != cudaSuccess || cudaEventCreate(&ev.b) != cudaSuccess))
        rc = fail(FW_ERR_CUDA, "event creation failed");
    unsigned int* bits = ctx->d_counter + 40;
    InvState* st = reinterpret_cast<InvState*>(ctx->d_scratch + SLOT_INV);
    // a smooth nonzero field for the gathers: the CC derivative of the pair, smoothed
    if (!rc) rc = launch_cc_pair_impl(ctx, fixed, moving, radius, a, b, ctx->d_scratch + SLOT_CC_VALUE, 0);
    if (!rc) rc = launch_smooth(ctx, a, u, variance, bits, e);
    if (!rc) rc = sync(ctx);
    // kinds 0-6 as documented; kind 4 includes the loop's init kernel, timed alone as kind 7 and
    // subtracted
    double t_init = 0.0;
    double deferred = 0.0;  // fraction of the step's tiles left to the fix kernel
    fw_invert_params once = {1, -1.0, -1.0, 1};
    for (int kind = 0; kind < 8 && !rc; ++kind) {
        auto launch = [&]() -> int {
            switch (kind) {
                case 0: return launch_warp(ctx, moving, u, nullptr, nullptr, out->d, false, nullptr);
                case 1: return launch_cc_pair_impl(ctx, fixed, moving, radius, a, b,
                                                   ctx->d_scratch + SLOT_CC_VALUE, 0);
                case 2: return launch_smooth(ctx, a, s, variance, bits, e);
                case 3: return launch_compose(ctx, u, w, w, bits, 0.1);
                case 4: {  // a first body of a fresh loop from a zero inverse
                    FW_TRY(enqueue_inversion_prefix(ctx, u, w, e, once, st, 0, 0));
                    return enqueue_inversion_body(ctx, u, w, e, st, 0, 0);
                }
                case 5: return enqueue_inversion_kernel(ctx, u, w, e, st, 0);
                case 6: return enqueue_inversion_kernel(ctx, u, w, e, st, 2);
                default: return enqueue_inversion_prefix(ctx, u, w, e, once, st, 0, 0);
            }
        };
        if (kind == 4 || kind == 5 || kind == 6) {  // every timed body starts from psi = 0
            FW_CUDA(cudaMemsetAsync(w->d, 0, w->bytes, ctx->stream));
        }
        if (kind == 5 || kind == 6) {  // a loop before its first body (and after its step)
            rc = enqueue_inversion_prefix(ctx, u, w, e, once, st, 0, 0);
            if (!rc && kind == 6) rc = enqueue_inversion_kernel(ctx, u, w, e, st, 0);
            if (!rc && kind == 6) rc = enqueue_inversion_kernel(ctx, u, w, e, st, 1);
            if (rc) break;
        }
        rc = launch();  // warm-up
        if (rc) break;
        if (kind == 6) {  // the step's deferred tiles, for the fix kernel's bytes
            InvState h;
            FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, st, sizeof(InvState), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            FW_TRY(sync(ctx));
            std::memcpy(&h, ctx->h_pinned, sizeof(h));
            deferred = (double)h.ndefer / (double)inv_step_parts(g);
        }
        cudaEventRecord(ev.a, ctx->stream);
        for (int r = 0; r < reps && !rc; ++r) rc = launch();
        cudaEventRecord(ev.b, ctx->stream);
        if (rc) break;
        rc = sync(ctx);
        float t = 0.0f;
        cudaEventElapsedTime(&t, ev.a, ev.b);
        if (kind < 7) ms[kind] = (double)t / reps;
        else t_init = (double)t / reps;
    }
    if (!rc) ms[4] = std::max(ms[4] - t_init, 1e-6);
    // algorithmic bytes: float32 voxels and field components
    bytes[0] = n * (12.0 + 4.0 + 4.0);         // field, source gather (one value), output
    bytes[1] = n * (8.0 + 24.0);               // two images in, two fields out
    bytes[2] = n * (12.0 + 12.0);              // field in, field out
    bytes[3] = n * (12.0 + 12.0 + 12.0);       // update gather, field in, field out
    bytes[4] = n * (12.0 + 12.0 + 12.0);       // psi in, field gather, psi out
    bytes[5] = (double)inv_bound_voxels(g) * 24.0;  // psi and the field gather on the lattice
    bytes[6] = deferred * n * 36.0;            // psi and residual in, psi out, deferred voxels
    fw_field_free(e);
    fw_field_free(u);
    fw_field_free(a);
    fw_field_free(b);
    fw_field_free(s);
    fw_field_free(w);
    fw_image_free(out);
    return rc;
}

}  // extern "C"
