// fw_prepare.cu -- the registration's image preparation on the device: isotropic resampling
// (crates/fastwarp-reg/src/register.rs:82-146) and antsRegistration's intensity preprocessing,
// a quantile window from a 256-bin histogram mapped onto [out_min, out_max]
// (crates/fastwarp-reg/src/preprocess.rs:45-215), composed as prepare_channels_with
// (register.rs:201-249).
//
// Both run once per image of a registration; they are HBM-bound passes over one image (the
// histogram needs the range first, so the preprocessing is three passes over the image: range,
// histogram, map; a one-block kernel walks the quantiles between the last two). Every result is bit-identical to the reference's f64 code for float32 input values:
// the arithmetic follows the reference's operation order with explicit round-to-nearest
// intrinsics (no fused multiply-add), the histogram counts are integers, and the quantile walk
// runs in one thread.
#include "fw_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace fw {
namespace {

constexpr int PRE_BINS = 256;          // preprocess.rs:36
constexpr double PRE_MARGIN = 10.0;    // preprocess.rs:37 (ITK's marginal scale)
constexpr int PRE_MAX_BLOCKS = 1024;

enum : int { PRE_OK = 0, PRE_NO_FINITE = 1, PRE_DEGENERATE = 2 };

// Device state of one preprocessing (zeroed before the first kernel).
struct PreState {
    double lo, hi;              // finite minimum and maximum
    double win_lo, win_hi;      // the quantile window, each a float32 value
    double scale, shift;        // the map inside the window
    unsigned long long finite;  // finite voxels
    int status;
    unsigned int counter_range;  // last-block counter
    unsigned int counts[PRE_BINS];
    float part_lo[PRE_MAX_BLOCKS], part_hi[PRE_MAX_BLOCKS];
    unsigned long long part_n[PRE_MAX_BLOCKS];
};

__device__ bool pre_last_block(unsigned int* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    return last;
}

__device__ __forceinline__ void pre_take(float v, float& lo, float& hi,
                                         unsigned long long& n) {
    if (isfinite(v)) {
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
        ++n;
    }
}

// preprocess.rs:48-61: minimum, maximum and count of the finite values.
__global__ void __launch_bounds__(256) k_pre_range(const float* __restrict__ x, long long n,
                                                   PreState* __restrict__ st) {
    float lo = INFINITY, hi = -INFINITY;
    unsigned long long cnt = 0;
    const long long n4 = n / 4;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long l = t0; l < n4; l += stride) {
        const float4 v = reinterpret_cast<const float4*>(x)[l];
        pre_take(v.x, lo, hi, cnt);
        pre_take(v.y, lo, hi, cnt);
        pre_take(v.z, lo, hi, cnt);
        pre_take(v.w, lo, hi, cnt);
    }
    for (long long l = 4 * n4 + t0; l < n; l += stride) pre_take(x[l], lo, hi, cnt);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    __shared__ float slo[8], shi[8];
    __shared__ unsigned long long sn[8];
    if ((threadIdx.x & 31) == 0) {
        slo[threadIdx.x >> 5] = lo;
        shi[threadIdx.x >> 5] = hi;
        sn[threadIdx.x >> 5] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            slo[0] = fminf(slo[0], slo[w]);
            shi[0] = fmaxf(shi[0], shi[w]);
            sn[0] += sn[w];
        }
        st->part_lo[blockIdx.x] = slo[0];
        st->part_hi[blockIdx.x] = shi[0];
        st->part_n[blockIdx.x] = sn[0];
    }
    if (!pre_last_block(&st->counter_range)) return;
    if (threadIdx.x == 0) {
        float a = INFINITY, b = -INFINITY;
        unsigned long long c = 0;
        for (unsigned int k = 0; k < gridDim.x; ++k) {
            a = fminf(a, __ldcg(st->part_lo + k));
            b = fmaxf(b, __ldcg(st->part_hi + k));
            c += __ldcg(st->part_n + k);
        }
        st->lo = a;
        st->hi = b;
        st->finite = c;
        st->status = c ? PRE_OK : PRE_NO_FINITE;
    }
}

// preprocess.rs:104-113: the bin whose lower edge is the last one <= v (the edges rise).
__device__ __forceinline__ int pre_bin(double v, const double* mn, double top) {
    if (v < mn[0]) return 0;
    if (v >= top) return PRE_BINS - 1;
    int lo = 0, hi = PRE_BINS;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (mn[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo > 0 ? lo - 1 : 0;
}

// preprocess.rs:115-161 (ITK Histogram::Quantile). mx[j] is mn[j + 1] below the last bin (the
// same expression) and `top` for the last.
__device__ double pre_quantile(const unsigned int* counts, const double* mn, double top,
                               double p) {
    double total = 0.0;
    for (int j = 0; j < PRE_BINS; ++j) total = __dadd_rn(total, (double)counts[j]);
    double cumulated = 0.0, p_prev = 0.0, f_n = 0.0;
    if (p < 0.5) {
        int n = 0;
        double p_n = 0.0;
        do {
            f_n = (double)counts[n];
            cumulated = __dadd_rn(cumulated, f_n);
            p_prev = p_n;
            p_n = __ddiv_rn(cumulated, total);
            ++n;
        } while (n < PRE_BINS && p_n < p);
        const double proportion = __ddiv_rn(f_n, total);
        const double lo = mn[n - 1];
        const double width = __dsub_rn(n < PRE_BINS ? mn[n] : top, lo);
        return __dadd_rn(lo, __dmul_rn(__ddiv_rn(__dsub_rn(p, p_prev), proportion), width));
    }
    int n = PRE_BINS - 1, m = 0;
    double p_n = 1.0;
    do {
        f_n = (double)counts[n];
        cumulated = __dadd_rn(cumulated, f_n);
        p_prev = p_n;
        p_n = __dsub_rn(1.0, __ddiv_rn(cumulated, total));
        --n;
        ++m;
    } while (m < PRE_BINS && p_n > p);
    const double proportion = __ddiv_rn(f_n, total);
    const int bin = n + 1;
    const double hi = bin + 1 < PRE_BINS ? mn[bin + 1] : top;
    const double width = __dsub_rn(hi, mn[bin]);
    return __dsub_rn(hi, __dmul_rn(__ddiv_rn(__dsub_rn(p_prev, p), proportion), width));
}

// preprocess.rs:62-77: ITK's float32 bin edges from the finite range (lower edges in `mn`, the
// last bin's upper edge in `top`, widened by a tenth of a bin). Every block builds the same table.
__device__ void pre_edges(const PreState* st, double* mn, double* top) {
    const double lo = st->lo, hi = st->hi;
    const double upper_edge = __dadd_rn(
        hi, __ddiv_rn(__ddiv_rn(__dsub_rn(hi, lo), (double)PRE_BINS), PRE_MARGIN));
    const float interval = __fdiv_rn(
        __fsub_rn(__double2float_rn(upper_edge), __double2float_rn(lo)), (float)PRE_BINS);
    for (int j = threadIdx.x; j < PRE_BINS; j += blockDim.x)
        mn[j] = __dadd_rn(lo, (double)__fmul_rn((float)j, interval));
    if (threadIdx.x == 0) *top = upper_edge;
}

// preprocess.rs:78-102: the histogram of the finite values (shared-memory counts per block,
// added into the global counts).
__global__ void __launch_bounds__(256) k_pre_hist(const float* __restrict__ x, long long n,
                                                  PreState* __restrict__ st) {
    __shared__ double mn[PRE_BINS];
    __shared__ unsigned int h[PRE_BINS];
    __shared__ double top;
    if (st->finite == 0) return;
    pre_edges(st, mn, &top);
    for (int j = threadIdx.x; j < PRE_BINS; j += blockDim.x) h[j] = 0;
    __syncthreads();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += stride) {
        const float v = x[l];
        if (isfinite(v)) atomicAdd(&h[pre_bin((double)v, mn, top)], 1u);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < PRE_BINS; j += blockDim.x)
        if (h[j]) atomicAdd(&st->counts[j], h[j]);
}

// preprocess.rs:168-209: both quantiles (one thread walks the counts), the degenerate-window
// test and the window map's scale and shift. One block.
__global__ void __launch_bounds__(256) k_pre_finish(PreState* __restrict__ st, float lower,
                                                    float upper, double out_min,
                                                    double out_max) {
    __shared__ double mn[PRE_BINS];
    __shared__ double top;
    if (st->finite == 0) return;
    pre_edges(st, mn, &top);
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double wl = (double)__double2float_rn(pre_quantile(st->counts, mn, top, (double)lower));
    const double wh = (double)__double2float_rn(pre_quantile(st->counts, mn, top, (double)upper));
    st->win_lo = wl;
    st->win_hi = wh;
    if (!(wh > wl)) {
        st->status = PRE_DEGENERATE;
        return;
    }
    const double scale = __ddiv_rn(__dsub_rn(out_max, out_min), __dsub_rn(wh, wl));
    st->scale = scale;
    st->shift = __dsub_rn(out_min, __dmul_rn(wl, scale));
}

// preprocess.rs:196-208 (IntensityWindowingTransform): below the window out_min, above it
// out_max, inside x * scale + shift; NaN passes through.
__global__ void __launch_bounds__(256) k_pre_window(const float* __restrict__ x,
                                                    float* __restrict__ out, long long n,
                                                    const PreState* __restrict__ st,
                                                    double out_min, double out_max) {
    if (st->status != PRE_OK) return;
    const double lo = st->win_lo, hi = st->win_hi, scale = st->scale, shift = st->shift;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += stride) {
        const double v = x[l];
        const double r = v < lo ? out_min : v > hi ? out_max : __dadd_rn(__dmul_rn(v, scale), shift);
        out[l] = __double2float_rn(r);
    }
}

struct IsoArgs {
    int sx, sy, sz;       // source size
    int ox, oy, oz;       // output size
    double ratio[3];      // mm / spacing
    double last[3];       // n - 1
};

// register.rs:82-108 and 130-143: output voxel (i, j, k) samples the source trilinearly at
// index min(i * ratio, n - 1) per axis, corners outside the buffer and zero weights skipped,
// summed in corner order, rounded to float32.
__global__ void __launch_bounds__(256) k_resample_iso(IsoArgs a, const float* __restrict__ src,
                                                      float* __restrict__ out) {
    const long long n = (long long)a.ox * a.oy * a.oz;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += stride) {
        const int i = (int)(l % a.ox);
        const int j = (int)((l / a.ox) % a.oy);
        const int k = (int)(l / ((long long)a.ox * a.oy));
        const double c[3] = {fmin(__dmul_rn((double)i, a.ratio[0]), a.last[0]),
                             fmin(__dmul_rn((double)j, a.ratio[1]), a.last[1]),
                             fmin(__dmul_rn((double)k, a.ratio[2]), a.last[2])};
        const double f[3] = {floor(c[0]), floor(c[1]), floor(c[2])};
        const double fr[3] = {__dsub_rn(c[0], f[0]), __dsub_rn(c[1], f[1]),
                              __dsub_rn(c[2], f[2])};
        const int base[3] = {(int)f[0], (int)f[1], (int)f[2]};
        const int size[3] = {a.sx, a.sy, a.sz};
        double acc = 0.0;
#pragma unroll
        for (int corner = 0; corner < 8; ++corner) {
            double w = 1.0;
            bool inside = true;
            int idx[3];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                const int bit = (corner >> ax) & 1;
                idx[ax] = base[ax] + bit;
                inside = inside && idx[ax] >= 0 && idx[ax] < size[ax];
                w = __dmul_rn(w, bit ? fr[ax] : __dsub_rn(1.0, fr[ax]));
            }
            if (!inside || w == 0.0) continue;
            const long long at = idx[0] + (long long)a.sx * (idx[1] + (long long)a.sy * idx[2]);
            acc = __dadd_rn(acc, __dmul_rn(w, (double)src[at]));
        }
        out[l] = __double2float_rn(acc);
    }
}

unsigned int pre_blocks(fw_ctx* ctx, long long n) {
    long long b = (n + 255) / 256;
    b = std::min<long long>(b, 4LL * ctx->num_sms);
    b = std::min<long long>(b, PRE_MAX_BLOCKS);
    return (unsigned int)std::max<long long>(b, 1);
}

// The header fields of PreState the host reads back.
struct PreHeader {
    double lo, hi, win_lo, win_hi, scale, shift;
    unsigned long long finite;
    int status;
};

int pre_state(fw_ctx* ctx, PreState** st) {
    FW_TRY(dev_alloc(ctx, sizeof(PreState), (void**)st));
    cudaError_t e = cudaMemsetAsync(*st, 0, sizeof(PreState), ctx->stream);
    if (e != cudaSuccess) {
        dev_free(ctx, *st, sizeof(PreState));
        return cuda_fail(e, "cudaMemsetAsync");
    }
    return 0;
}

int pre_read(fw_ctx* ctx, PreState* st, PreHeader* out) {
    static_assert(sizeof(PreHeader) <= 4096 * sizeof(double), "pinned read-back space");
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, st, sizeof(PreHeader), cudaMemcpyDeviceToHost,
                            ctx->stream));
    FW_TRY(sync(ctx));
    ctx->stats.bytes_downloaded += sizeof(PreHeader);
    std::memcpy(out, ctx->h_pinned, sizeof(PreHeader));
    return 0;
}

// Counts the finite voxels of an image.
int count_finite(fw_ctx* ctx, const fw_image* img, unsigned long long* finite) {
    const long long n = img->grid.count();
    PreState* st;
    FW_TRY(pre_state(ctx, &st));
    k_pre_range<<<pre_blocks(ctx, n), 256, 0, ctx->stream>>>(img->d, n, st);
    int rc = check_launch(ctx, "k_pre_range");
    PreHeader h{};
    if (!rc) rc = pre_read(ctx, st, &h);
    dev_free(ctx, st, sizeof(PreState));
    if (!rc) *finite = h.finite;
    return rc;
}

// preprocess_values (preprocess.rs:180-209); `out` may be null (the window only).
int preprocess(fw_ctx* ctx, const fw_image* img, float lower, float upper, double out_min,
               double out_max, fw_image* out, double window[2]) {
    const long long n = img->grid.count();
    PreState* st;
    FW_TRY(pre_state(ctx, &st));
    const unsigned int blocks = pre_blocks(ctx, n);
    k_pre_range<<<blocks, 256, 0, ctx->stream>>>(img->d, n, st);
    int rc = check_launch(ctx, "k_pre_range");
    if (!rc) {
        k_pre_hist<<<blocks, 256, 0, ctx->stream>>>(img->d, n, st);
        rc = check_launch(ctx, "k_pre_hist");
    }
    if (!rc) {
        k_pre_finish<<<1, 256, 0, ctx->stream>>>(st, lower, upper, out_min, out_max);
        rc = check_launch(ctx, "k_pre_finish");
    }
    if (!rc && out) {
        k_pre_window<<<blocks, 256, 0, ctx->stream>>>(img->d, out->d, n, st, out_min, out_max);
        rc = check_launch(ctx, "k_pre_window");
    }
    PreHeader h{};
    if (!rc) rc = pre_read(ctx, st, &h);
    dev_free(ctx, st, sizeof(PreState));
    if (rc) return rc;
    if (h.status == PRE_NO_FINITE)
        return fail(FW_ERR_INVALID, "preprocess: image has no finite values");
    if (window) {
        window[0] = h.win_lo;
        window[1] = h.win_hi;
    }
    if (h.status == PRE_DEGENERATE) {
        char msg[160];
        std::snprintf(msg, sizeof(msg), "preprocess: degenerate intensity window [%.17g, %.17g]",
                      h.win_lo, h.win_hi);
        return fail(FW_ERR_INVALID, msg);
    }
    return 0;
}

bool same_spacing(const HostGrid& g, double mm) {
    for (int a = 0; a < 3; ++a)
        if (!(std::fabs(g.sp[a] - mm) < 1e-6)) return false;
    return true;
}

int copy_image(fw_ctx* ctx, const fw_image* img, fw_image** out) {
    fw_image* im;
    FW_TRY(new_image(ctx, img->grid, &im));
    cudaError_t e = cudaMemcpyAsync(im->d, img->d, img->grid.count() * sizeof(float),
                                    cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) {
        fw_image_free(im);
        return cuda_fail(e, "cudaMemcpyAsync");
    }
    *out = im;
    return 0;
}

// resample_isotropic (register.rs:112-146): a new image on the isotropic grid, or a copy.
int resample_isotropic(fw_ctx* ctx, const fw_image* img, double mm, fw_image** out) {
    FW_CHECK(std::isfinite(mm) && mm > 0.0, "isotropic spacing must be positive");
    const HostGrid& g = img->grid;
    if (same_spacing(g, mm)) return copy_image(ctx, img, out);
    fw_image* im;
    IsoArgs a{};
    fw_grid og = to_c(g);
    for (int ax = 0; ax < 3; ++ax) {
        a.last[ax] = (double)(g.n[ax] - 1);
        a.ratio[ax] = mm / g.sp[ax];
        const double t = std::floor(a.last[ax] * g.sp[ax] / mm + 1e-9);
        FW_CHECK(t < 2147483647.0, "grid too large: 2^31 voxels or more");
        og.size[ax] = std::max<int64_t>((int64_t)t + 1, 1);
        og.spacing[ax] = mm;
    }
    HostGrid hg;
    FW_TRY(make_grid(&og, hg));
    a.sx = (int)g.n[0];
    a.sy = (int)g.n[1];
    a.sz = (int)g.n[2];
    a.ox = (int)hg.n[0];
    a.oy = (int)hg.n[1];
    a.oz = (int)hg.n[2];
    FW_TRY(new_image(ctx, hg, &im));
    const long long n = hg.count();
    const unsigned int blocks =
        (unsigned int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 16LL * ctx->num_sms));
    k_resample_iso<<<blocks, 256, 0, ctx->stream>>>(a, img->d, im->d);
    int rc = check_launch(ctx, "k_resample_iso");
    if (rc) {
        fw_image_free(im);
        return rc;
    }
    *out = im;
    return 0;
}

}  // namespace
}  // namespace fw

using namespace fw;

extern "C" {

int fw_quantile_window(fw_ctx* ctx, const fw_image* img, float lower, float upper,
                       double window[2]) {
    FW_CHECK(ctx && img && window, "null argument");
    return preprocess(ctx, img, lower, upper, 0.0, 1.0, nullptr, window);
}

int fw_preprocess(fw_ctx* ctx, const fw_image* img, float lower, float upper, double out_min,
                  double out_max, fw_image** out, double window[2]) {
    FW_CHECK(ctx && img && out, "null argument");
    *out = nullptr;
    fw_image* im;
    FW_TRY(new_image(ctx, img->grid, &im));
    int rc = preprocess(ctx, img, lower, upper, out_min, out_max, im, window);
    if (rc) {
        fw_image_free(im);
        return rc;
    }
    *out = im;
    return 0;
}

int fw_resample_isotropic(fw_ctx* ctx, const fw_image* img, double mm, fw_image** out) {
    FW_CHECK(ctx && img && out, "null argument");
    *out = nullptr;
    fw_image* im;
    FW_TRY(resample_isotropic(ctx, img, mm, &im));
    int rc = sync(ctx);
    if (rc) {
        fw_image_free(im);
        return rc;
    }
    *out = im;
    return 0;
}

int fw_prepare_channels(fw_ctx* ctx, int32_t channels, const fw_image* const* fixed,
                        const fw_image* const* moving, const double* iso_mm,
                        const float* winsorize, fw_image** fixed_out, fw_image** moving_out,
                        fw_image** fixed_raw, fw_image** moving_raw) {
    FW_CHECK(ctx && fixed_out && moving_out, "null argument");
    float lower = 0.0f, upper = 1.0f;
    if (winsorize) {
        lower = winsorize[0];
        upper = winsorize[1];
        FW_CHECK(0.0f <= lower && lower < upper && upper <= 1.0f,
                 "winsorize must be (lower, upper) quantiles with 0 <= lower < upper <= 1");
    }
    FW_CHECK(channels > 0 && fixed && moving,
             "fixed and moving must have the same, non-zero number of channels");
    for (int32_t c = 0; c < channels; ++c) {
        fixed_out[c] = moving_out[c] = nullptr;
        if (fixed_raw) fixed_raw[c] = nullptr;
        if (moving_raw) moving_raw[c] = nullptr;
    }
    for (int32_t c = 0; c < channels; ++c)
        FW_CHECK(fixed[c] && moving[c], "null image");
    for (int s = 0; s < 2; ++s)
        for (int32_t c = 0; c < channels; ++c) {
            const fw_image* im = s ? moving[c] : fixed[c];
            unsigned long long finite = 0;
            FW_TRY(count_finite(ctx, im, &finite));
            FW_CHECK(finite == (unsigned long long)im->grid.count(),
                     "an input image has non-finite (NaN or infinite) voxels");
        }
    if (iso_mm) FW_CHECK(std::isfinite(*iso_mm) && *iso_mm > 0.0,
                         "isotropic spacing must be positive");
    std::vector<fw_image*> raw(2 * (size_t)channels, nullptr), done(2 * (size_t)channels, nullptr);
    auto release = [&](int rc) {
        for (fw_image* im : raw) if (im) fw_image_free(im);
        for (fw_image* im : done) if (im) fw_image_free(im);
        return rc;
    };
    int rc = 0;
    for (int s = 0; s < 2 && !rc; ++s)
        for (int32_t c = 0; c < channels && !rc; ++c) {
            const fw_image* im = s ? moving[c] : fixed[c];
            fw_image*& r = raw[(size_t)s * channels + c];
            rc = iso_mm ? resample_isotropic(ctx, im, *iso_mm, &r) : copy_image(ctx, im, &r);
        }
    for (int32_t c = 0; c < channels && !rc; ++c)
        for (int s = 0; s < 2 && !rc; ++s) {
            const size_t k = (size_t)s * channels + c;
            rc = new_image(ctx, raw[k]->grid, &done[k]);
            if (!rc) rc = preprocess(ctx, raw[k], lower, upper, 0.0, 1.0, done[k], nullptr);
        }
    if (rc) return release(rc);
    for (int32_t c = 0; c < channels; ++c) {
        fixed_out[c] = done[c];
        moving_out[c] = done[(size_t)channels + c];
        done[c] = done[(size_t)channels + c] = nullptr;
        if (fixed_raw) {
            fixed_raw[c] = raw[c];
            raw[c] = nullptr;
        }
        if (moving_raw) {
            moving_raw[c] = raw[(size_t)channels + c];
            raw[(size_t)channels + c] = nullptr;
        }
    }
    return release(0);
}

}  // extern "C"
