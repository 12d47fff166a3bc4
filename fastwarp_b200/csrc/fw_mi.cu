// fw_mi.cu -- sampled Mattes mutual information of the Rigid/Affine stages: the joint Parzen
// histogram, ITK's ComputeResults and the parameter gradient (metric/mi.rs:364-511, 702-768;
// GPU counterpart GpuMiLevel, crates/fastwarp-gpu/src/wgpu_backend/mi.rs:144-491).
//
// Device design:
//  - samples are resident as 16-byte records (x, y, z relative to the cloud centre as float32,
//    fixed bin as u32): one vector load per sample;
//  - the histogram is accumulated in 2^-32 fixed point as u64 in block-private shared memory
//    and merged with u64 atomics: integer sums do not depend on order, so a rerun is
//    bit-identical, and the normalising sum is exact (no Kahan sum needed);
//  - ComputeResults (normalisation, marginals, -MI, the per-cell ratio) runs on the device in
//    float64, one thread per cell, so value_and_derivative needs a single read-back;
//  - the derivative is linear in the Jacobian, which is affine in the sample point for Euler3D and
//    affine transforms: col_mu(p) = G_mu [p; 1]. The kernel therefore reduces only the twelve
//    moments M_ij = sum_s w_s grad_i(s) [r_s; 1]_j (w_s = sum_k B3'(k - term) ratio[f, k]) and the
//    host contracts them with every parameter's G_mu in float64 -- the same sum as the
//    reference's sum_cell dpdf[cell] * ratio[cell], reordered.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <vector>

#include "fw_internal.cuh"

struct fw_mi_level {
    fw_ctx* ctx;
    fw_image* moving;
    bool own_moving;
    bool own_rec;  // false: the records belong to the caller (a linear chain's sample cache)
    float4* d_rec;
    int64_t n;
    double center[3];
    fw_mi_binning binning;
    unsigned long long* d_hist;  // [T][bins*bins + bins]
    double* d_ratio;             // [bins*bins]
    double* d_out;               // [T][4]: value, num_valid, status, pad
    double* d_mom;               // [12]
    double* d_part;              // block partials
    unsigned int* d_counter;
    unsigned int blocks;
    unsigned int hist_grid;  // resident histogram blocks (one wave)
    size_t hist_smem;
    bool hist_clear;         // the histograms are zero (the next pass may add into them)
    int64_t last_valid;
    size_t rec_bytes;
};

namespace fw {

namespace {

constexpr int MI_THREADS = 256;
constexpr int MAX_BINS = 32;  // one thread per joint cell in k_mi_finish
constexpr double FIXED = 4294967296.0;  // 2^32

struct MiMap {
    double a[9];   // moving index from relative sample point
    double b[3];
    double h[3][3];  // index offset of +half a spacing along physical axis d (central difference)
    DevGrid m;
    int bins;
    double mmin, mmax, mbin, mnmin;
};

__device__ __forceinline__ double bspline3(double u) {
    double a = fabs(u);
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

__device__ __forceinline__ double bspline3_derivative(double u) {
    if (u >= 0.0 && u < 1.0) return -2.0 * u + 1.5 * u * u;
    if (u > -1.0 && u < 0.0) return -2.0 * u - 1.5 * u * u;
    if (u >= 1.0 && u < 2.0) return -2.0 + 2.0 * u - 0.5 * u * u;
    if (u > -2.0 && u <= -1.0) return 2.0 + 2.0 * u + 0.5 * u * u;
    return 0.0;
}

__device__ __forceinline__ int clamp_bin(double term, int bins) {
    long long idx = isnan(term) ? 0 : (long long)term;  // truncation toward zero
    return (int)min(max(idx, 2LL), (long long)bins - 3);
}

// The moving sample: index, interpolated value and its Parzen term; false when the sample does
// not contribute (outside the buffer, not finite, or outside the moving range).
__device__ __forceinline__ bool sample_value(const MiMap& mp, const float* __restrict__ img,
                                             float4 r, double c[3], double& mv, double& term,
                                             int& mbin) {
#pragma unroll
    for (int q = 0; q < 3; ++q)
        c[q] = mp.a[q * 3] * r.x + mp.a[q * 3 + 1] * r.y + mp.a[q * 3 + 2] * r.z + mp.b[q];
    if (!inside_index(c[0], c[1], c[2], mp.m.nx, mp.m.ny, mp.m.nz)) return false;
    float v = lin_at_index(img, mp.m.nx, mp.m.ny, mp.m.nz, c[0], c[1], c[2]);
    mv = (double)v;
    if (!isfinite(v) || mv < mp.mmin || mv > mp.mmax) return false;
    term = mv / mp.mbin - mp.mnmin;
    mbin = clamp_bin(term, mp.bins);
    return true;
}

// Copies of the histogram per block: lane l adds into copy l mod MI_REP, so one warp instruction
// puts at most 32 / MI_REP lanes on any cell (neighbouring samples see nearly the same
// intensities and would otherwise all hit one cell); each copy is padded by one cell so a cell's
// copies lie on different shared-memory banks. Integer sums: the merged histogram is exact.
constexpr int MI_REP = 8;

size_t mi_hist_smem(int bins) {
    return sizeof(unsigned long long) * MI_REP * (size_t)(bins * bins + bins + 1);
}

// Joint histogram of one transform over a chunk of samples per block, added into `out`.
__device__ __forceinline__ void mi_hist_body(const MiMap& mp, const float4* __restrict__ rec,
                                             long long n, const float* __restrict__ img,
                                             unsigned long long* __restrict__ out) {
    const int bins = mp.bins;
    const int cells = bins * bins + bins;
    const int cstride = cells + 1;
    extern __shared__ unsigned long long sh_all[];
    for (int s = threadIdx.x; s < MI_REP * cstride; s += blockDim.x) sh_all[s] = 0ULL;
    __syncthreads();
    unsigned long long* sh = sh_all + (threadIdx.x & (MI_REP - 1)) * cstride;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float4 r = __ldg(rec + i);
        double c[3], mv, term;
        int mbin;
        if (!sample_value(mp, img, r, c, mv, term, mbin)) continue;
        const int fbin = (int)__float_as_uint(r.w);
        atomicAdd(&sh[bins * bins + fbin], 1ULL);
#pragma unroll
        for (int pm = -1; pm <= 2; ++pm) {
            double w = bspline3((double)(mbin + pm) - term);
            unsigned long long q = (unsigned long long)__double2ll_rn(w * FIXED);
            if (q) atomicAdd(&sh[fbin * bins + mbin + pm], q);
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < cells; s += blockDim.x) {
        unsigned long long v = 0ULL;
#pragma unroll
        for (int k = 0; k < MI_REP; ++k) v += sh_all[k * cstride + s];
        if (v) atomicAdd(&out[s], v);
    }
}

// Transform blockIdx.y of a batch (maps in device memory).
__global__ void __launch_bounds__(MI_THREADS) k_mi_hist(const MiMap* __restrict__ maps,
                                                        const float4* __restrict__ rec,
                                                        long long n,
                                                        const float* __restrict__ img,
                                                        unsigned long long* __restrict__ hist) {
    const MiMap& mp = maps[blockIdx.y];
    mi_hist_body(mp, rec, n, img, hist + (size_t)blockIdx.y * (mp.bins * mp.bins + mp.bins));
}

// One transform, its map passed with the launch (no copy ahead of it).
__global__ void __launch_bounds__(MI_THREADS) k_mi_hist1(const __grid_constant__ MiMap mp,
                                                         const float4* __restrict__ rec,
                                                         long long n,
                                                         const float* __restrict__ img,
                                                         unsigned long long* __restrict__ hist) {
    mi_hist_body(mp, rec, n, img, hist);
}

// ComputeResults (metric/mi.rs:702-768) for histogram blockIdx.x: one thread per cell.
// out[t*4 + 0] = -MI, [1] = valid samples, [2] = status (0 ok, 1 no valid sample, 2 zero PDF);
// ratio[t * bins * bins + cell] with want_ratio. The moving bin size is `moving_bin_size`, or
// mbin_dev[t] when that is given (bin sizes measured on the device). With `clear` the histogram
// is zeroed once read, ready for the next evaluation's pass.
__device__ __forceinline__ void mi_finish_body(const unsigned long long* h, int bins,
                                               double moving_bin_size, double* ratio, double* o,
                                               int want_ratio);

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(1024) k_mi_finish(unsigned long long* hist, int bins,
                                                    double moving_bin_size,
                                                    const double* __restrict__ mbin_dev,
                                                    double* __restrict__ ratio_all,
                                                    double* __restrict__ out, int want_ratio,
                                                    int clear) {
    const int cells = bins * bins + bins;
    unsigned long long* h = hist + (size_t)blockIdx.x * cells;
    if (mbin_dev) moving_bin_size = mbin_dev[blockIdx.x];
    mi_finish_body(h, bins, moving_bin_size, ratio_all + (size_t)blockIdx.x * bins * bins,
                   out + 4 * blockIdx.x, want_ratio);
    if (clear) {
        __syncthreads();  // every read of the histogram is done
        for (int s = threadIdx.x; s < cells; s += blockDim.x) h[s] = 0ULL;
    }
}

__device__ __forceinline__ void mi_finish_body(const unsigned long long* h, int bins,
                                               double moving_bin_size, double* ratio, double* o,
                                               int want_ratio) {
    __shared__ unsigned long long s_js[32], s_vs[32];
    __shared__ double s_c[32];
    __shared__ double fmarg[MAX_BINS], mmarg[MAX_BINS];
    __shared__ double norm_s;
    __shared__ unsigned long long valid_s;
    const int t = threadIdx.x, lane = t & 31, wp = t >> 5, nw = blockDim.x >> 5;
    const int nc = bins * bins;
    // exact integer totals: the joint sum and the number of valid samples (warp shuffles, then
    // the first warp over the warps' sums)
    unsigned long long js = 0, vs = 0;
    for (int s = t; s < nc; s += blockDim.x) js += h[s];
    for (int s = t; s < bins; s += blockDim.x) vs += h[nc + s];
    js = warp_sum_u64(js);
    vs = warp_sum_u64(vs);
    if (lane == 0) {
        s_js[wp] = js;
        s_vs[wp] = vs;
    }
    __syncthreads();
    if (wp == 0) {
        unsigned long long a = lane < nw ? s_js[lane] : 0ULL, b = lane < nw ? s_vs[lane] : 0ULL;
        a = warp_sum_u64(a);
        b = warp_sum_u64(b);
        if (lane == 0) {
            norm_s = (double)a / FIXED;
            valid_s = b;
        }
    }
    __syncthreads();
    const double pdf_sum = norm_s;
    const unsigned long long num_valid = valid_s;
    if (num_valid == 0 || pdf_sum < DBL_EPSILON) {
        if (t == 0) {
            o[0] = 0.0;
            o[1] = (double)num_valid;
            o[2] = num_valid == 0 ? 1.0 : 2.0;
        }
        return;
    }
    const double norm = 1.0 / pdf_sum;
    if (t < bins) fmarg[t] = (double)h[nc + t] * norm;
    if (t < bins) {
        double s = 0.0;
        for (int row = 0; row < bins; ++row) s += ((double)h[row * bins + t] / FIXED) * norm;
        mmarg[t] = s;
    }
    __syncthreads();
    const double n_factor = -1.0 / (moving_bin_size * (double)num_valid);
    double contrib = 0.0;
    if (t < nc) {
        int f = t / bins, m = t - f * bins;
        double fm = fmarg[f], mm = mmarg[m];
        double jv = ((double)h[t] / FIXED) * norm;
        double r = 0.0;
        if (fm > DBL_EPSILON && mm > DBL_EPSILON && jv > DBL_EPSILON) {
            double pr = log(jv / mm);
            contrib = jv * (pr - log(fm));
            r = n_factor * pr;
        }
        if (want_ratio) ratio[t] = r;
    }
    // the sum of the cells' terms in a fixed order: each warp's butterfly, then the first warp's
    // over the warps in order
    contrib = warp_sum_d(contrib);
    if (lane == 0) s_c[wp] = contrib;
    __syncthreads();
    double total = 0.0;
    if (wp == 0) total = warp_sum_d(lane < nw ? s_c[lane] : 0.0);
    if (t == 0) {
        o[0] = -total;
        o[1] = (double)num_valid;
        o[2] = 0.0;
    }
}

// Derivative moments M[i][j] = sum_s w_s grad_i [r; 1]_j with a fixed-order last-block reduction.
__global__ void __launch_bounds__(MI_THREADS, 3) k_mi_deriv(const __grid_constant__ MiMap mp,
                                                         const float4* __restrict__ rec,
                                                         long long n,
                                                         const float* __restrict__ img,
                                                         const double* __restrict__ ratio,
                                                         double* __restrict__ partials,
                                                         unsigned int* __restrict__ counter,
                                                         double* __restrict__ mom) {
    const int bins = mp.bins;
    __shared__ double sratio[MAX_BINS * MAX_BINS];
    for (int s = threadIdx.x; s < bins * bins; s += blockDim.x) sratio[s] = ratio[s];
    __syncthreads();
    double acc[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) acc[q] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float4 r = __ldg(rec + i);
        double c[3], mv, term;
        int mbin;
        if (!sample_value(mp, img, r, c, mv, term, mbin)) continue;
        const int fbin = (int)__float_as_uint(r.w);
        double w = 0.0;
#pragma unroll
        for (int pm = -1; pm <= 2; ++pm)
            w += bspline3_derivative((double)(mbin + pm) - term) * sratio[fbin * bins + mbin + pm];
        if (w == 0.0) continue;
        // interp.rs:96-120: half-spacing central difference along the physical axes. All six
        // probes are interpolated unconditionally (lin_at_index clamps every corner into the
        // buffer), so their 48 loads can be in flight together; an axis with a probe outside the
        // buffer then contributes zero, as the reference's early exit does.
        double g[3];
        float v1[3], v2[3];
        bool ok[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double c1x = c[0] - mp.h[d][0], c1y = c[1] - mp.h[d][1], c1z = c[2] - mp.h[d][2];
            const double c2x = c[0] + mp.h[d][0], c2y = c[1] + mp.h[d][1], c2z = c[2] + mp.h[d][2];
            ok[d] = inside_index(c1x, c1y, c1z, mp.m.nx, mp.m.ny, mp.m.nz) &&
                    inside_index(c2x, c2y, c2z, mp.m.nx, mp.m.ny, mp.m.nz);
            v1[d] = lin_at_index(img, mp.m.nx, mp.m.ny, mp.m.nz, c1x, c1y, c1z);
            v2[d] = lin_at_index(img, mp.m.nx, mp.m.ny, mp.m.nz, c2x, c2y, c2z);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) g[d] = ok[d] ? (double)(v2[d] - v1[d]) / mp.m.sp[d] : 0.0;
        if (!(isfinite(g[0]) && isfinite(g[1]) && isfinite(g[2]))) g[0] = g[1] = g[2] = 0.0;
        const double p[4] = {(double)r.x, (double)r.y, (double)r.z, 1.0};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a * 4 + b] += w * g[a] * p[b];
    }
    __shared__ double red[12][MI_THREADS / 32];
    __shared__ bool last;
#pragma unroll
    for (int q = 0; q < 12; ++q) {
        double v = warp_sum_d(acc[q]);
        if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        double s = 0.0;
        for (int w = 0; w < MI_THREADS / 32; ++w) s += red[threadIdx.x][w];
        partials[(size_t)blockIdx.x * 12 + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    // the whole last block sums the partials of each moment in a fixed order
    __shared__ double fin[MI_THREADS / 32];
    for (int q = 0; q < 12; ++q) {
        const double s = block_sum_fixed(partials + q, gridDim.x, 12, fin);
        if (threadIdx.x == 0) mom[q] = s;
    }
    if (threadIdx.x == 0) *counter = 0;
}

// ---- dense Mattes MI pair of two images on one grid (SyN Mattes channels) -----------------
//
// Backend::mi_value_derivative_pair[_masked] (backend.rs:179-205) as cpu/mod.rs:352-381 runs it:
// MattesMi::evaluate_dense (metric/mi.rs:601-680) twice, (fixed, moving) then (moving, fixed),
// with identity transforms and the masks (when given) on the images' grid. Both directions use
// the same two Parzen terms per voxel (f / s_f - n_f and m / s_m - n_m), so one pass builds both
// joint histograms and one pass writes both derivatives. The intensity ranges (MiBinning::dense,
// mi.rs:276-295: each image over the voxels inside its own mask, non-finite voxels skipped) and
// the bin geometry (MiBinning::from_ranges, mi.rs:238-274) are measured on the device.

struct DenseState {
    unsigned int key[4];    // order-preserving keys of f min, f max, m min, m max
    unsigned int count[2];  // finite voxels inside each image's own mask
    int status;             // 0 ok; 1 / 2 no finite fixed / moving voxel; 3 / 4 constant
    int pad;
    double fmin, fmax, mmin, mmax;
    double sf, nf, sm, nm;  // bin size and normalised minimum of each image
    double mbin[2];         // moving-axis bin size of direction 0 (m) and 1 (f)
};

__device__ __forceinline__ unsigned int order_key(float v) {
    unsigned int b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ float key_value(unsigned int k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void k_dense_init(DenseState* st) {
    st->key[0] = st->key[2] = 0xffffffffu;
    st->key[1] = st->key[3] = 0u;
    st->count[0] = st->count[1] = 0u;
    st->status = 0;
}

__global__ void __launch_bounds__(256) k_dense_range(const float* __restrict__ f,
                                                     const float* __restrict__ m,
                                                     const float* __restrict__ fm,
                                                     const float* __restrict__ mm, long long n,
                                                     DenseState* __restrict__ st) {
    unsigned int kl[2] = {0xffffffffu, 0xffffffffu}, kh[2] = {0u, 0u}, cnt[2] = {0u, 0u};
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < n;
         l += (long long)gridDim.x * blockDim.x) {
        const float v[2] = {f[l], m[l]};
        const bool in[2] = {!fm || fm[l] != 0.0f, !mm || mm[l] != 0.0f};
#pragma unroll
        for (int q = 0; q < 2; ++q)
            if (in[q] && isfinite(v[q])) {
                const unsigned int k = order_key(v[q]);
                kl[q] = min(kl[q], k);
                kh[q] = max(kh[q], k);
                ++cnt[q];
            }
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            kl[q] = min(kl[q], __shfl_xor_sync(0xffffffffu, kl[q], o));
            kh[q] = max(kh[q], __shfl_xor_sync(0xffffffffu, kh[q], o));
            cnt[q] += __shfl_xor_sync(0xffffffffu, cnt[q], o);
        }
        if ((threadIdx.x & 31) == 0 && cnt[q]) {
            atomicMin(&st->key[2 * q], kl[q]);
            atomicMax(&st->key[2 * q + 1], kh[q]);
            atomicAdd(&st->count[q], cnt[q]);
        }
    }
}

__global__ void k_dense_setup(DenseState* st, int bins) {
    if (st->count[0] == 0) {
        st->status = 1;
        return;
    }
    if (st->count[1] == 0) {
        st->status = 2;
        return;
    }
    st->fmin = key_value(st->key[0]);
    st->fmax = key_value(st->key[1]);
    st->mmin = key_value(st->key[2]);
    st->mmax = key_value(st->key[3]);
    if (st->fmax - st->fmin <= DBL_EPSILON) {
        st->status = 3;
        return;
    }
    if (st->mmax - st->mmin <= DBL_EPSILON) {
        st->status = 4;
        return;
    }
    const double span = (double)(bins - 4);
    st->sf = (st->fmax - st->fmin) / span;
    st->sm = (st->mmax - st->mmin) / span;
    st->nf = st->fmin / st->sf - 2.0;
    st->nm = st->mmin / st->sm - 2.0;
    st->mbin[0] = st->sm;
    st->mbin[1] = st->sf;
}

// The voxel's two Parzen terms and bins; false when it does not contribute (mi.rs:560-595).
__device__ __forceinline__ bool dense_voxel(const DenseState& st, int bins, float a, float b,
                                            bool in, double& tf, double& tm, int& bf, int& bm) {
    if (!in || !isfinite(a) || !isfinite(b)) return false;
    const double fv = a, mv = b;
    // each direction's moving value must lie in its range: m for (f, m), f for (m, f)
    if (mv < st.mmin || mv > st.mmax || fv < st.fmin || fv > st.fmax) return false;
    tf = fv / st.sf - st.nf;
    tm = mv / st.sm - st.nm;
    bf = clamp_bin(tf, bins);
    bm = clamp_bin(tm, bins);
    return true;
}

// Copies of the pair's two histograms per block (lane l into copy l mod MI_REP_DENSE).
constexpr int MI_REP_DENSE = 4;

size_t dense_hist_smem(int bins) {
    return sizeof(unsigned long long) * MI_REP_DENSE * (size_t)(2 * (bins * bins + bins) + 1);
}

// Both joint histograms: [direction][bins*bins joint + bins fixed marginal] in 2^-32 fixed point.
__global__ void __launch_bounds__(MI_THREADS) k_dense_hist(const float* __restrict__ f,
                                                           const float* __restrict__ m,
                                                           const float* __restrict__ fm,
                                                           const float* __restrict__ mm,
                                                           long long n, int bins,
                                                           const DenseState* __restrict__ st,
                                                           unsigned long long* __restrict__ hist) {
    extern __shared__ unsigned long long sh_all[];
    const int nc = bins * bins, cells = nc + bins;
    const int cstride = 2 * cells + 1;  // copies as in k_mi_hist, padded onto different banks
    for (int s = threadIdx.x; s < MI_REP_DENSE * cstride; s += blockDim.x) sh_all[s] = 0ULL;
    __syncthreads();
    unsigned long long* sh = sh_all + (threadIdx.x & (MI_REP_DENSE - 1)) * cstride;
    const DenseState S = *st;
    if (S.status == 0) {
        for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < n;
             l += (long long)gridDim.x * blockDim.x) {
            double tf, tm;
            int bf, bm;
            const bool in = (!fm || fm[l] != 0.0f) && (!mm || mm[l] != 0.0f);
            if (!dense_voxel(S, bins, f[l], m[l], in, tf, tm, bf, bm)) continue;
            atomicAdd(&sh[nc + bf], 1ULL);
            atomicAdd(&sh[cells + nc + bm], 1ULL);
#pragma unroll
            for (int k = -1; k <= 2; ++k) {
                unsigned long long q0 =
                    (unsigned long long)__double2ll_rn(bspline3((double)(bm + k) - tm) * FIXED);
                unsigned long long q1 =
                    (unsigned long long)__double2ll_rn(bspline3((double)(bf + k) - tf) * FIXED);
                if (q0) atomicAdd(&sh[bf * bins + bm + k], q0);
                if (q1) atomicAdd(&sh[cells + bm * bins + bf + k], q1);
            }
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < 2 * cells; s += blockDim.x) {
        unsigned long long v = 0ULL;
#pragma unroll
        for (int k = 0; k < MI_REP_DENSE; ++k) v += sh_all[k * cstride + s];
        if (v) atomicAdd(&hist[s], v);
    }
}

struct DenseArgs {
    DevGrid g;
    long long ps;
    int bins;
    int identity;
    double isp[3];
};

// Both derivatives (mi.rs:655-672): sum_k B3'(k - term) ratio[fixed bin, k] * grad(moving image of
// the direction), zero where the voxel does not contribute; result[0..1] = their sums of squares.
__global__ void __launch_bounds__(MI_THREADS) k_dense_deriv(
    DenseArgs a, const float* __restrict__ f, const float* __restrict__ m,
    const float* __restrict__ fm, const float* __restrict__ mm, const DenseState* __restrict__ st,
    const double* __restrict__ ratio, float* __restrict__ d0, float* __restrict__ d1,
    double* __restrict__ partials, unsigned int* __restrict__ counter,
    double* __restrict__ result) {
    __shared__ double sr[2 * MAX_BINS * MAX_BINS];
    const int bins = a.bins, nc = bins * bins;
    for (int s = threadIdx.x; s < 2 * nc; s += blockDim.x) sr[s] = ratio[s];
    __syncthreads();
    const DenseState S = *st;
    double n0 = 0.0, n1 = 0.0;
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < a.g.n;
         l += (long long)gridDim.x * blockDim.x) {
        double tf, tm;
        int bf, bm;
        const bool in = (!fm || fm[l] != 0.0f) && (!mm || mm[l] != 0.0f);
        float o0[3] = {0.0f, 0.0f, 0.0f}, o1[3] = {0.0f, 0.0f, 0.0f};
        if (S.status == 0 && dense_voxel(S, bins, f[l], m[l], in, tf, tm, bf, bm)) {
            double w0 = 0.0, w1 = 0.0;
#pragma unroll
            for (int k = -1; k <= 2; ++k) {
                w0 += bspline3_derivative((double)(bm + k) - tm) * sr[bf * bins + bm + k];
                w1 += bspline3_derivative((double)(bf + k) - tf) * sr[nc + bm * bins + bf + k];
            }
            int i, j, kz;
            voxel_ijk(l, a.g.nx, a.g.ny, i, j, kz);
            float gm[3], gf[3];
            central_difference_voxel(m, a.g, a.identity != 0, a.isp, i, j, kz, gm);
            central_difference_voxel(f, a.g, a.identity != 0, a.isp, i, j, kz, gf);
            if (!(isfinite(gm[0]) && isfinite(gm[1]) && isfinite(gm[2]))) gm[0] = gm[1] = gm[2] = 0.0f;
            if (!(isfinite(gf[0]) && isfinite(gf[1]) && isfinite(gf[2]))) gf[0] = gf[1] = gf[2] = 0.0f;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                o0[d] = (float)(w0 * (double)gm[d]);
                o1[d] = (float)(w1 * (double)gf[d]);
                n0 += (double)o0[d] * o0[d];
                n1 += (double)o1[d] * o1[d];
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            d0[l + d * a.ps] = o0[d];
            d1[l + d * a.ps] = o1[d];
        }
    }
    __shared__ double red[2][MI_THREADS / 32];
    __shared__ bool last;
    n0 = warp_sum_d(n0);
    n1 = warp_sum_d(n1);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = n0;
        red[1][threadIdx.x >> 5] = n1;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int w = 0; w < MI_THREADS / 32; ++w) s += red[threadIdx.x][w];
        partials[(size_t)blockIdx.x * 2 + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __shared__ double fin[MI_THREADS / 32];
    for (int q = 0; q < 2; ++q) {
        const double s = block_sum_fixed(partials + q, gridDim.x, 2, fin);
        if (threadIdx.x == 0) result[q] = s;
    }
    if (threadIdx.x == 0) *counter = 0;
}

// ---- host: transform maps and Jacobian matrices (transform/param.rs, affine.rs) -------------

void parametric_affine(const fw_linear_transform* t, double M[9], double off[3]) {
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

void linear_map(const fw_linear_transform* t, double Mout[9], double off_out[3]) {
    double M[9], off[3];
    parametric_affine(t, M, off);
    double oc[3], ooff[3];
    mat3_vec(t->outer_matrix, t->outer_center, oc);
    for (int r = 0; r < 3; ++r) ooff[r] = t->outer_translation[r] + t->outer_center[r] - oc[r];
    mat3_mul(t->outer_matrix, M, Mout);
    double mo[3];
    mat3_vec(t->outer_matrix, off, mo);
    for (int r = 0; r < 3; ++r) off_out[r] = mo[r] + ooff[r];
}

// transform/param.rs:188-288, 448-457: Jacobian columns at p (outer matrix applied).
int jacobian_columns(const fw_linear_transform* t, const double p[3], double cols[36]) {
    for (int k = 0; k < 36; ++k) cols[k] = 0.0;
    int np;
    if (t->kind == 0) {
        const double* q = t->parameters;
        double cx = std::cos(q[0]), sx = std::sin(q[0]);
        double cy = std::cos(q[1]), sy = std::sin(q[1]);
        double cz = std::cos(q[2]), sz = std::sin(q[2]);
        double px = p[0] - t->center[0], py = p[1] - t->center[1], pz = p[2] - t->center[2];
        double *o0 = cols, *o1 = cols + 3, *o2 = cols + 6;
        if (t->zyx) {
            o0[0] = (cz * sy * cx + sz * sx) * py + (-cz * sy * sx + sz * cx) * pz;
            o0[1] = (sz * sy * cx - cz * sx) * py + (-sz * sy * sx - cz * cx) * pz;
            o0[2] = (cy * cx) * py + (-cy * sx) * pz;
            o1[0] = (-cz * sy) * px + (cz * cy * sx) * py + (cz * cy * cx) * pz;
            o1[1] = (-sz * sy) * px + (sz * cy * sx) * py + (sz * cy * cx) * pz;
            o1[2] = (-cy) * px + (-sy * sx) * py + (-sy * cx) * pz;
            o2[0] = (-sz * cy) * px + (-sz * sy * sx - cz * cx) * py + (-sz * sy * cx + cz * sx) * pz;
            o2[1] = (cz * cy) * px + (cz * sy * sx - sz * cx) * py + (cz * sy * cx + sz * sx) * pz;
        } else {
            o0[0] = (-sz * cx * sy) * px + (sz * sx) * py + (sz * cx * cy) * pz;
            o0[1] = (cz * cx * sy) * px + (-cz * sx) * py + (-cz * cx * cy) * pz;
            o0[2] = (sx * sy) * px + cx * py + (-sx * cy) * pz;
            o1[0] = (-cz * sy - sz * sx * cy) * px + (cz * cy - sz * sx * sy) * pz;
            o1[1] = (-sz * sy + cz * sx * cy) * px + (sz * cy + cz * sx * sy) * pz;
            o1[2] = (-cx * cy) * px + (-cx * sy) * pz;
            o2[0] = (-sz * cy - cz * sx * sy) * px + (-cz * cx) * py + (-sz * sy + cz * sx * cy) * pz;
            o2[1] = (cz * cy - sz * sx * sy) * px + (-sz * cx) * py + (cz * sy + sz * sx * cy) * pz;
        }
        for (int d = 0; d < 3; ++d) cols[3 * (3 + d) + d] = 1.0;
        np = 6;
    } else {
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) cols[3 * (r * 3 + c) + r] = p[c] - t->center[c];
            cols[3 * (9 + r) + r] = 1.0;
        }
        np = 12;
    }
    for (int k = 0; k < np; ++k) {
        double v[3] = {cols[3 * k], cols[3 * k + 1], cols[3 * k + 2]}, o[3];
        mat3_vec(t->outer_matrix, v, o);
        for (int r = 0; r < 3; ++r) cols[3 * k + r] = o[r];
    }
    return np;
}

MiMap make_map(const fw_mi_level* L, const fw_linear_transform* t) {
    MiMap mp;
    std::memset(&mp, 0, sizeof(mp));
    const HostGrid& g = L->moving->grid;
    double M[9], off[3];
    linear_map(t, M, off);
    // index = inv (M (centre + r) + off - org) = (inv M) r + inv (M centre + off - org)
    mat3_mul(g.inv, M, mp.a);
    double mc[3];
    mat3_vec(M, L->center, mc);
    double v[3] = {mc[0] + off[0] - g.org[0], mc[1] + off[1] - g.org[1], mc[2] + off[2] - g.org[2]};
    mat3_vec(g.inv, v, mp.b);
    for (int d = 0; d < 3; ++d)
        for (int r = 0; r < 3; ++r) mp.h[d][r] = 0.5 * g.sp[d] * g.inv[r * 3 + d];
    mp.m = dev_grid(g);
    mp.bins = L->binning.bins;
    mp.mmin = L->binning.moving_min;
    mp.mmax = L->binning.moving_max;
    mp.mbin = L->binning.moving_bin_size;
    mp.mnmin = L->binning.moving_normalized_min;
    return mp;
}

// The histogram kernel's shared memory can exceed the 48 KB default.
int hist_launch_setup(fw_ctx* ctx, size_t smem) {
    (void)ctx;
    FW_CUDA(cudaFuncSetAttribute(k_mi_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FW_CUDA(cudaFuncSetAttribute(k_mi_hist1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return 0;
}

// One wave of resident histogram blocks (each merges its copies into the global histogram once).
unsigned int hist_blocks(const fw_mi_level* L, size_t smem) {
    int occ = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mi_hist, MI_THREADS, smem) != cudaSuccess ||
        occ < 1) {
        cudaGetLastError();
        occ = 1;
    }
    const long long want = (L->n + MI_THREADS - 1) / MI_THREADS;
    return (unsigned int)std::max<long long>(1, std::min<long long>(want, (long long)occ * L->ctx->num_sms));
}

// The histogram pass and ComputeResults of `count` transforms. One transform's map goes with
// the launch; a batch's maps are copied ahead. The histograms are zero before the pass (cleared
// by the previous ComputeResults, or here after an interrupted evaluation) and cleared again by
// this one's. `map0` (nullable) receives the first transform's map.
int hist_and_finish(fw_mi_level* L, const fw_linear_transform* ts, int count, bool want_ratio,
                    MiMap* map0 = nullptr) {
    fw_ctx* ctx = L->ctx;
    const int bins = L->binning.bins;
    const int cells = bins * bins + bins;
    if (!L->hist_clear) {
        FW_CUDA(cudaMemsetAsync(L->d_hist, 0, sizeof(unsigned long long) * cells * 16, ctx->stream));
        L->hist_clear = true;
    }
    L->hist_clear = false;
    if (count == 1) {
        const MiMap mp = make_map(L, &ts[0]);
        if (map0) *map0 = mp;
        k_mi_hist1<<<L->hist_grid, MI_THREADS, L->hist_smem, ctx->stream>>>(mp, L->d_rec, L->n,
                                                                             L->moving->d, L->d_hist);
        FW_TRY(check_launch(ctx, "k_mi_hist1"));
    } else {
        std::vector<MiMap> maps(count);
        for (int t = 0; t < count; ++t) maps[t] = make_map(L, &ts[t]);
        if (map0) *map0 = maps[0];
        FW_TRY(ensure_scratch(ctx, SLOT_PARTIALS + (sizeof(MiMap) * count + 7) / 8 + 16));
        MiMap* d_maps = reinterpret_cast<MiMap*>(ctx->d_scratch + SLOT_PARTIALS);
        FW_CUDA(cudaMemcpyAsync(d_maps, maps.data(), sizeof(MiMap) * count, cudaMemcpyHostToDevice,
                                ctx->stream));
        dim3 grid(L->hist_grid, count);
        k_mi_hist<<<grid, MI_THREADS, L->hist_smem, ctx->stream>>>(d_maps, L->d_rec, L->n,
                                                                  L->moving->d, L->d_hist);
        FW_TRY(check_launch(ctx, "k_mi_hist"));
    }
    k_mi_finish<<<count, 1024, 0, ctx->stream>>>(L->d_hist, bins, L->binning.moving_bin_size,
                                                 nullptr, L->d_ratio, L->d_out,
                                                 want_ratio ? 1 : 0, 1);
    FW_TRY(check_launch(ctx, "k_mi_finish"));
    L->hist_clear = true;
    return 0;
}

int check_status(fw_mi_level* L, const double* out) {
    L->last_valid = (int64_t)out[1];
    if (out[2] == 1.0) return fail(FW_ERR_INVALID, "mattes: all samples map outside the moving image buffer");
    if (out[2] == 2.0) return fail(FW_ERR_INVALID, "mattes: joint PDF summed to zero");
    return 0;
}

}  // namespace

}  // namespace fw

using namespace fw;

// A level over sample records already on the device (float32 offsets from `center`, the fixed
// bin in w). Takes the moving image when own_moving and the records when own_rec, also on failure.
int fw::mi_level_create(fw_ctx* ctx, fw_image* moving, bool own_moving, float4* d_rec,
                        bool own_rec, int64_t n, const double center[3],
                        const fw_mi_binning* binning, fw_mi_level** out) {
    auto drop = [&] {
        if (own_rec && d_rec) dev_free(ctx, d_rec, sizeof(float4) * (size_t)std::max<int64_t>(n, 0));
        if (own_moving) fw_image_free(moving);
    };
    if (n <= 0) {
        drop();
        return fail(FW_ERR_INVALID, "mattes: no samples inside the fixed image");
    }
    if (binning->bins <= 4 || binning->bins > MAX_BINS) {
        drop();
        return fail(FW_ERR_INVALID, "mattes: bins must be in 5..=32");
    }
    fw_mi_level* L = new fw_mi_level();
    L->ctx = ctx;
    L->moving = moving;
    L->own_moving = own_moving;
    L->own_rec = own_rec;
    L->d_rec = d_rec;
    L->n = n;
    L->binning = *binning;
    for (int a = 0; a < 3; ++a) L->center[a] = center[a];
    L->rec_bytes = sizeof(float4) * (size_t)n;
    const int cells = binning->bins * binning->bins + binning->bins;
    const int max_t = 16;
    // the gradient pass: one wave of resident blocks (a partial second wave would run its tail
    // at a fraction of the occupancy)
    int occ = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mi_deriv, MI_THREADS, 0) != cudaSuccess ||
        occ < 1) {
        cudaGetLastError();
        occ = 1;
    }
    L->blocks = (unsigned int)std::max<long long>(
        1, std::min<long long>((n + MI_THREADS - 1) / MI_THREADS, (long long)occ * ctx->num_sms));
    int rc = dev_alloc(ctx, sizeof(unsigned long long) * cells * max_t, (void**)&L->d_hist);
    if (!rc) rc = dev_alloc(ctx, sizeof(double) * binning->bins * binning->bins, (void**)&L->d_ratio);
    if (!rc) rc = dev_alloc(ctx, sizeof(double) * 4 * max_t, (void**)&L->d_out);
    if (!rc) rc = dev_alloc(ctx, sizeof(double) * 16, (void**)&L->d_mom);
    if (!rc) rc = dev_alloc(ctx, sizeof(double) * 12 * L->blocks, (void**)&L->d_part);
    if (!rc) rc = dev_alloc(ctx, sizeof(unsigned int) * 4, (void**)&L->d_counter);
    if (!rc) {
        cudaError_t e = cudaMemsetAsync(L->d_counter, 0, sizeof(unsigned int) * 4, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(L->d_hist, 0, sizeof(unsigned long long) * cells * max_t, ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "mi level setup");
        L->hist_clear = true;
    }
    if (!rc) {
        L->hist_smem = mi_hist_smem(binning->bins);
        rc = hist_launch_setup(ctx, L->hist_smem);
        if (!rc) L->hist_grid = hist_blocks(L, L->hist_smem);
    }
    if (rc) {
        fw_mi_level_free(L);
        return rc;
    }
    *out = L;
    return 0;
}

extern "C" {

static int mi_prepare_common(fw_ctx* ctx, fw_image* moving, bool own, const double* points,
                             const uint32_t* fixed_bin, int64_t n, const fw_mi_binning* binning,
                             fw_mi_level** out) {
    if (n <= 0 || binning->bins <= 4 || binning->bins > MAX_BINS)
        return mi_level_create(ctx, moving, own, nullptr, false, n, nullptr, binning, out);
    // the cloud centre in float64; records hold float32 offsets from it
    double c[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) c[a] += points[3 * i + a];
    for (int a = 0; a < 3; ++a) c[a] /= (double)n;
    std::vector<float4> rec((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        if (fixed_bin[i] >= (uint32_t)binning->bins) {
            if (own) fw_image_free(moving);
            return fail(FW_ERR_INVALID, "mattes: a fixed bin is out of range");
        }
        rec[i].x = (float)(points[3 * i] - c[0]);
        rec[i].y = (float)(points[3 * i + 1] - c[1]);
        rec[i].z = (float)(points[3 * i + 2] - c[2]);
        uint32_t b = fixed_bin[i];
        std::memcpy(&rec[i].w, &b, 4);
    }
    const size_t bytes = sizeof(float4) * (size_t)n;
    float4* d_rec = nullptr;
    int rc = dev_alloc(ctx, bytes, (void**)&d_rec);
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(d_rec, rec.data(), bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "mi level upload");
        ctx->stats.bytes_uploaded += bytes;
    }
    if (!rc) rc = sync(ctx);
    if (rc) {
        if (d_rec) dev_free(ctx, d_rec, bytes);
        if (own) fw_image_free(moving);
        return rc;
    }
    return mi_level_create(ctx, moving, own, d_rec, true, n, c, binning, out);
}

int fw_mi_level_prepare(fw_ctx* ctx, const fw_grid* moving_grid, const double* moving,
                        const double* points, const uint32_t* fixed_bin, int64_t n,
                        const fw_mi_binning* binning, fw_mi_level** out) {
    FW_CHECK(ctx && moving_grid && moving && points && fixed_bin && binning && out, "null argument");
    fw_image* img;
    FW_TRY(fw_image_upload(ctx, moving_grid, moving, &img));
    return mi_prepare_common(ctx, img, true, points, fixed_bin, n, binning, out);
}

int fw_mi_level_prepare_image(fw_ctx* ctx, const fw_image* moving, const double* points,
                              const uint32_t* fixed_bin, int64_t n,
                              const fw_mi_binning* binning, fw_mi_level** out) {
    FW_CHECK(ctx && moving && points && fixed_bin && binning && out, "null argument");
    return mi_prepare_common(ctx, const_cast<fw_image*>(moving), false, points, fixed_bin, n,
                             binning, out);
}

int fw_mi_level_value(fw_mi_level* L, const fw_linear_transform* t, double* value) {
    FW_CHECK(L && t && value, "null argument");
    FW_TRY(hist_and_finish(L, t, 1, false));
    double out[3];
    FW_TRY(read_back(L->ctx, L->d_out, 3, out));
    FW_TRY(check_status(L, out));
    *value = out[0];
    return 0;
}

int fw_mi_level_values(fw_mi_level* L, const fw_linear_transform* ts, int32_t count,
                       double* values) {
    FW_CHECK(L && ts && values, "null argument");
    FW_CHECK(count >= 1 && count <= 16, "mattes: 1..=16 transforms per batch");
    FW_TRY(hist_and_finish(L, ts, count, false));
    std::vector<double> out(4 * count);
    FW_TRY(read_back(L->ctx, L->d_out, 4 * count, out.data()));
    for (int t = 0; t < count; ++t) {
        FW_TRY(check_status(L, &out[4 * t]));
        values[t] = out[4 * t];
    }
    return 0;
}

int fw_mi_level_value_and_derivative(fw_mi_level* L, const fw_linear_transform* t,
                                     double* value, double* derivative) {
    FW_CHECK(L && t && value && derivative, "null argument");
    fw_ctx* ctx = L->ctx;
    MiMap mp;
    FW_TRY(hist_and_finish(L, t, 1, true, &mp));
    k_mi_deriv<<<L->blocks, MI_THREADS, 0, ctx->stream>>>(mp, L->d_rec, L->n, L->moving->d,
                                                          L->d_ratio, L->d_part, L->d_counter,
                                                          L->d_mom);
    FW_TRY(check_launch(ctx, "k_mi_deriv"));
    // one read-back: status block (value, valid, status) and the twelve moments
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, L->d_out, sizeof(double) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned + 4, L->d_mom, sizeof(double) * 12, cudaMemcpyDeviceToHost, ctx->stream));
    FW_TRY(sync(ctx));
    double out[4], mom[12];
    std::memcpy(out, ctx->h_pinned, sizeof(out));
    std::memcpy(mom, ctx->h_pinned + 4, sizeof(mom));
    FW_TRY(check_status(L, out));
    *value = out[0];
    // G_mu in relative coordinates: col_mu(c + r) = J(c) + (J(c + e_j) - J(c)) r_j
    double j0[36], je[3][36];
    FW_TRY(0);
    int np = jacobian_columns(t, L->center, j0);
    for (int j = 0; j < 3; ++j) {
        double p[3] = {L->center[0], L->center[1], L->center[2]};
        p[j] += 1.0;
        jacobian_columns(t, p, je[j]);
    }
    for (int mu = 0; mu < np; ++mu) {
        double s = 0.0;
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) s += (je[j][3 * mu + i] - j0[3 * mu + i]) * mom[i * 4 + j];
            s += j0[3 * mu + i] * mom[i * 4 + 3];
        }
        derivative[mu] = s;
    }
    return 0;
}

int fw_mi_level_time(fw_mi_level* L, const fw_linear_transform* t, int32_t reps, double ms[3],
                     double bytes[3]) {
    FW_CHECK(L && t && ms && bytes && reps > 0, "null argument");
    fw_ctx* ctx = L->ctx;
    // one evaluation first: the maps in scratch, the ratio table and the status
    double v = 0.0, d[12];
    FW_TRY(fw_mi_level_value_and_derivative(L, t, &v, d));
    const int bins = L->binning.bins;
    const int cells = bins * bins + bins;
    const MiMap mp = make_map(L, t);
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        if (a) cudaEventDestroy(a);
        return fail(FW_ERR_CUDA, "event creation failed");
    }
    int rc = 0;
    for (int kind = 0; kind < 3 && !rc; ++kind) {
        auto launch = [&]() -> int {
            if (kind == 0) {
                FW_CUDA(cudaMemsetAsync(L->d_hist, 0, sizeof(unsigned long long) * cells,
                                        ctx->stream));
                k_mi_hist1<<<L->hist_grid, MI_THREADS, L->hist_smem, ctx->stream>>>(
                    mp, L->d_rec, L->n, L->moving->d, L->d_hist);
                return check_launch(ctx, "k_mi_hist1");
            }
            if (kind == 1) {
                k_mi_finish<<<1, 1024, 0, ctx->stream>>>(L->d_hist, bins, L->binning.moving_bin_size,
                                                         nullptr, L->d_ratio, L->d_out, 1, 0);
                return check_launch(ctx, "k_mi_finish");
            }
            k_mi_deriv<<<L->blocks, MI_THREADS, 0, ctx->stream>>>(mp, L->d_rec, L->n,
                                                                  L->moving->d, L->d_ratio,
                                                                  L->d_part, L->d_counter,
                                                                  L->d_mom);
            return check_launch(ctx, "k_mi_deriv");
        };
        rc = launch();  // warm-up
        if (rc) break;
        cudaEventRecord(a, ctx->stream);
        for (int r = 0; r < reps && !rc; ++r) rc = launch();
        cudaEventRecord(b, ctx->stream);
        if (!rc) rc = sync(ctx);
        float tm = 0.0f;
        if (!rc) cudaEventElapsedTime(&tm, a, b);
        ms[kind] = (double)tm / reps;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    L->hist_clear = false;  // the timed passes leave a histogram behind
    // algorithmic bytes per pass: the 16-byte sample records plus the moving image's gathers,
    // at most the whole image and at most one 8-corner gather per sample (32 bytes)
    const double S = (double)L->n, Nm = (double)L->moving->grid.count();
    const double pass = 16.0 * S + std::min(4.0 * Nm, 32.0 * S);
    bytes[0] = pass + 8.0 * cells;
    bytes[1] = 16.0 * cells;
    bytes[2] = pass + 8.0 * bins * bins;
    return rc;
}

int fw_mi_level_num_valid(const fw_mi_level* L, int64_t* out) {
    FW_CHECK(L && out, "null argument");
    *out = L->last_valid;
    return 0;
}

int fw_mi_level_samples(const fw_mi_level* L, double* points, uint32_t* fixed_bins, int64_t cap,
                        int64_t* n, fw_mi_binning* binning) {
    FW_CHECK(L && n, "null argument");
    *n = L->n;
    if (binning) *binning = L->binning;
    if (cap < L->n || (!points && !fixed_bins)) return 0;
    fw_ctx* ctx = L->ctx;
    std::vector<float4> rec((size_t)L->n);
    FW_CUDA(cudaMemcpyAsync(rec.data(), L->d_rec, L->rec_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    FW_TRY(sync(ctx));
    ctx->stats.bytes_downloaded += L->rec_bytes;
    for (int64_t i = 0; i < L->n; ++i) {
        if (points) {
            points[3 * i] = L->center[0] + (double)rec[i].x;
            points[3 * i + 1] = L->center[1] + (double)rec[i].y;
            points[3 * i + 2] = L->center[2] + (double)rec[i].z;
        }
        if (fixed_bins) std::memcpy(&fixed_bins[i], &rec[i].w, 4);
    }
    return 0;
}

void fw_mi_level_free(fw_mi_level* L) {
    if (!L) return;
    fw_ctx* ctx = L->ctx;
    const int cells = L->binning.bins * L->binning.bins + L->binning.bins;
    if (L->own_rec) dev_free(ctx, L->d_rec, L->rec_bytes);
    dev_free(ctx, L->d_hist, sizeof(unsigned long long) * cells * 16);
    dev_free(ctx, L->d_ratio, sizeof(double) * L->binning.bins * L->binning.bins);
    dev_free(ctx, L->d_out, sizeof(double) * 4 * 16);
    dev_free(ctx, L->d_mom, sizeof(double) * 16);
    dev_free(ctx, L->d_part, sizeof(double) * 12 * L->blocks);
    dev_free(ctx, L->d_counter, sizeof(unsigned int) * 4);
    if (L->own_moving) fw_image_free(L->moving);
    delete L;
}

}  // extern "C"

namespace fw {
void linear_transform_map(const fw_linear_transform* t, double M[9], double off[3]) {
    linear_map(t, M, off);
}

const fw_ctx* mi_level_context(const fw_mi_level* level) { return level ? level->ctx : nullptr; }
}  // namespace fw

// ---- dense Mattes MI pair: host side -----------------------------------------------------------

namespace fw {
namespace {

std::string empty_range_message(const char* role, bool masked) {
    if (masked)
        return std::string("no finite ") + role + "-image voxel lies inside the " + role + " mask";
    return std::string("the ") + role + " image has no finite voxel";
}

// [vF, |dF|^2, |dM|^2, 0, vM, status]: the scalars of one pair where the SyN driver reads them.
// status: 0 ok, 1 / 2 no finite fixed / moving voxel (inside its mask), 3 / 4 fixed / moving
// image constant, 5 no voxel contributes, 6 joint PDF zero.
__global__ void k_dense_publish(const DenseState* __restrict__ st, const double* __restrict__ out,
                                const double* __restrict__ norms, double* __restrict__ pub) {
    int status = st->status;
    for (int dir = 0; dir < 2 && status == 0; ++dir) {
        if (out[4 * dir + 2] == 1.0) status = 5;
        else if (out[4 * dir + 2] == 2.0) status = 6;
    }
    pub[0] = out[0];
    pub[1] = norms[0];
    pub[2] = norms[1];
    pub[3] = 0.0;
    pub[4] = out[4];
    pub[5] = (double)status;
}

}  // namespace
}  // namespace fw

// Device scratch of one dense pair: [state | out 2x4 | norms 2 | hist | ratio | partials].
struct fw_dense_mi {
    fw_ctx* ctx = nullptr;
    void* base = nullptr;
    size_t bytes = 0;
    int bins = 0;
    unsigned int blocks = 0;
    fw::DenseState* st = nullptr;
    double* out = nullptr;
    double* norms = nullptr;
    unsigned long long* hist = nullptr;
    double* ratio = nullptr;
    double* partials = nullptr;
    unsigned int* counter = nullptr;
};

namespace fw {

int dense_mi_create(fw_ctx* ctx, int bins, long long n, fw_dense_mi** out) {
    if (bins <= 4) return fail(FW_ERR_INVALID, "mattes: at least five histogram bins are required");
    if (bins > MAX_BINS) return fail(FW_ERR_INVALID, "mattes: bins must be in 5..=32");
    fw_dense_mi* d = new fw_dense_mi();
    d->ctx = ctx;
    d->bins = bins;
    d->blocks = (unsigned int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 2LL * ctx->num_sms));
    const size_t cells = (size_t)bins * bins + bins;
    const size_t o_hist = 512, o_ratio = o_hist + 16 * cells,
                 o_part = o_ratio + 16 * (size_t)bins * bins, o_cnt = o_part + 16 * (size_t)d->blocks;
    d->bytes = o_cnt + 256;
    int rc = dev_alloc(ctx, d->bytes, &d->base);
    if (rc) {
        delete d;
        return rc;
    }
    char* b = static_cast<char*>(d->base);
    d->st = reinterpret_cast<DenseState*>(b);
    d->out = reinterpret_cast<double*>(b + 256);
    d->norms = reinterpret_cast<double*>(b + 256 + 64);
    d->hist = reinterpret_cast<unsigned long long*>(b + o_hist);
    d->ratio = reinterpret_cast<double*>(b + o_ratio);
    d->partials = reinterpret_cast<double*>(b + o_part);
    d->counter = reinterpret_cast<unsigned int*>(b + o_cnt);
    cudaError_t e = cudaMemsetAsync(d->base, 0, d->bytes, ctx->stream);
    if (e != cudaSuccess) {
        dense_mi_free(d);
        return cuda_fail(e, "dense MI scratch");
    }
    *out = d;
    return 0;
}

void dense_mi_free(fw_dense_mi* d) {
    if (!d) return;
    if (d->base) dev_free(d->ctx, d->base, d->bytes);
    delete d;
}

int enqueue_dense_mi_pair(fw_ctx* ctx, const fw_image* f, const fw_image* m, const fw_image* fm,
                          const fw_image* mm, fw_field* d_fixed, fw_field* d_moving,
                          fw_dense_mi* sc, double* publish) {
    if (!f->grid.same(m->grid)) return fail(FW_ERR_INVALID, "mattes: the images are not on one grid");
    if ((fm && !fm->grid.same(f->grid)) || (mm && !mm->grid.same(f->grid)))
        return fail(FW_ERR_INVALID, "mattes: a mask is not on the grid of the images");
    const HostGrid& g = f->grid;
    const long long n = g.count();
    const int bins = sc->bins;
    const unsigned int blocks = sc->blocks;
    const float* fmp = fm ? fm->d : nullptr;
    const float* mmp = mm ? mm->d : nullptr;
    k_dense_init<<<1, 1, 0, ctx->stream>>>(sc->st);
    FW_TRY(check_launch(ctx, "k_dense_init"));
    FW_CUDA(cudaMemsetAsync(sc->hist, 0, 16 * ((size_t)bins * bins + bins), ctx->stream));
    k_dense_range<<<blocks, 256, 0, ctx->stream>>>(f->d, m->d, fmp, mmp, n, sc->st);
    FW_TRY(check_launch(ctx, "k_dense_range"));
    k_dense_setup<<<1, 1, 0, ctx->stream>>>(sc->st, bins);
    FW_TRY(check_launch(ctx, "k_dense_setup"));
    const size_t sh = dense_hist_smem(bins);
    FW_CUDA(cudaFuncSetAttribute(k_dense_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
    k_dense_hist<<<blocks, MI_THREADS, sh, ctx->stream>>>(f->d, m->d, fmp, mmp, n, bins, sc->st,
                                                          sc->hist);
    FW_TRY(check_launch(ctx, "k_dense_hist"));
    k_mi_finish<<<2, 1024, 0, ctx->stream>>>(sc->hist, bins, 0.0, sc->st->mbin, sc->ratio,
                                             sc->out, 1, 0);
    FW_TRY(check_launch(ctx, "k_mi_finish"));
    DenseArgs da;
    std::memset(&da, 0, sizeof(da));
    da.g = dev_grid(g);
    da.ps = d_fixed->ps;
    da.bins = bins;
    da.identity = 1;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            if (g.dir[r * 3 + c] != (r == c ? 1.0 : 0.0)) da.identity = 0;
    for (int d = 0; d < 3; ++d) da.isp[d] = 1.0 / g.sp[d];
    k_dense_deriv<<<blocks, MI_THREADS, 0, ctx->stream>>>(da, f->d, m->d, fmp, mmp, sc->st,
                                                          sc->ratio, d_fixed->d, d_moving->d,
                                                          sc->partials, sc->counter, sc->norms);
    FW_TRY(check_launch(ctx, "k_dense_deriv"));
    k_dense_publish<<<1, 1, 0, ctx->stream>>>(sc->st, sc->out, sc->norms, publish);
    return check_launch(ctx, "k_dense_publish");
}

int dense_mi_status(int status, bool masked) {
    switch (status) {
        case 0: return 0;
        case 1: return fail(FW_ERR_INVALID, "mattes: " + empty_range_message("fixed", masked));
        case 2: return fail(FW_ERR_INVALID, "mattes: " + empty_range_message("moving", masked));
        case 3: return fail(FW_ERR_INVALID, "mattes: the fixed image is constant");
        case 4: return fail(FW_ERR_INVALID, "mattes: the moving image is constant");
        case 5:
            return fail(FW_ERR_INVALID, masked ? std::string("mattes: ") + FW_NO_VOXEL_IN_MASKS
                                               : std::string("mattes: all samples map outside the moving image buffer"));
        default: return fail(FW_ERR_INVALID, "mattes: joint PDF summed to zero");
    }
}

namespace {

int dense_pair(fw_ctx* ctx, const fw_image* f, const fw_image* m, const fw_image* fm,
               const fw_image* mm, int bins, double values[2], fw_field** d_fixed,
               fw_field** d_moving, double norms[2]) {
    FW_CHECK(ctx && f && m && values && d_fixed && d_moving, "null argument");
    if (!f->grid.same(m->grid)) return fail(FW_ERR_INVALID, "mattes: the images are not on one grid");
    fw_dense_mi* sc = nullptr;
    FW_TRY(dense_mi_create(ctx, bins, f->grid.count(), &sc));
    fw_field *a = nullptr, *b = nullptr;
    int rc = new_field(ctx, f->grid, &a);
    if (!rc) rc = new_field(ctx, f->grid, &b);
    double* pub = ctx->d_scratch + SLOT_MI;
    if (!rc) rc = enqueue_dense_mi_pair(ctx, f, m, fm, mm, a, b, sc, pub);
    double h[6] = {0, 0, 0, 0, 0, 0};
    if (!rc) rc = read_back(ctx, pub, 6, h);
    if (!rc) rc = dense_mi_status((int)h[5], fm || mm);
    dense_mi_free(sc);
    if (rc) {
        fw_field_free(a);
        fw_field_free(b);
        return rc;
    }
    values[0] = h[0];
    values[1] = h[4];
    if (norms) {
        norms[0] = std::sqrt(h[1]);
        norms[1] = std::sqrt(h[2]);
    }
    *d_fixed = a;
    *d_moving = b;
    return 0;
}

}  // namespace
}  // namespace fw

extern "C" {

int fw_mi_value_derivative_pair(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                                int32_t bins, double values[2], fw_field** d_fixed,
                                fw_field** d_moving) {
    return fw::dense_pair(ctx, fixed, moving, nullptr, nullptr, bins, values, d_fixed, d_moving,
                          nullptr);
}

int fw_mi_value_derivative_pair_masked(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                                       const fw_image* fixed_mask, const fw_image* moving_mask,
                                       int32_t bins, double values[2], fw_field** d_fixed,
                                       fw_field** d_moving) {
    return fw::dense_pair(ctx, fixed, moving, fixed_mask, moving_mask, bins, values, d_fixed,
                          d_moving, nullptr);
}

int fw_mi_value_derivative_pair_with_norms(fw_ctx* ctx, const fw_image* fixed,
                                           const fw_image* moving, int32_t bins, double values[2],
                                           fw_field** d_fixed, fw_field** d_moving,
                                           double norms[2]) {
    FW_CHECK(norms, "null norms");
    return fw::dense_pair(ctx, fixed, moving, nullptr, nullptr, bins, values, d_fixed, d_moving,
                          norms);
}

int fw_mi_value_derivative_pair_masked_with_norms(fw_ctx* ctx, const fw_image* fixed,
                                                  const fw_image* moving,
                                                  const fw_image* fixed_mask,
                                                  const fw_image* moving_mask, int32_t bins,
                                                  double values[2], fw_field** d_fixed,
                                                  fw_field** d_moving, double norms[2]) {
    FW_CHECK(norms, "null norms");
    return fw::dense_pair(ctx, fixed, moving, fixed_mask, moving_mask, bins, values, d_fixed,
                          d_moving, norms);
}

}  // extern "C"
