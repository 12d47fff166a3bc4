// fw_cc.cu -- ANTs neighbourhood cross-correlation, both directions in one pass.
//
// Restates metric/cc.rs:170-321 (CcMetric::evaluate_masked with identity transforms on one grid,
// what cpu/mod.rs:299-331 runs for Backend::cc_value_derivative_pair): the six window sums over a
// clamped (2r+1)^3 box, local CC = sFM^2 / (sFF sMM), value = -mean(localCC), and the derivative
// coefficient * grad(moving) by ITK's half-spacing central difference (interp.rs:96-120).
//
// Kernel design (sm_100a): one CTA owns a TX x TY column tile and marches along z over a chunk
// of slices. Each input slice (with an r-voxel halo in x and y) is staged in shared memory; the
// x and y box passes run in shared memory and the z window is a running sum over a ring of the
// per-slice xy sums. Sums are float64: products of float32 voxels are exact in float64, so the
// centred second moments (sum f^2 - (sum f)^2 / n) keep their precision in flat bright regions
// where float32 cancels. The window planes never touch HBM: the kernel reads the two images once
// (plus halo re-reads that hit L2) and writes the two derivative fields.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>

#include "fw_internal.cuh"

namespace fw {

namespace {

constexpr int TX = 32;

struct CcArgs {
    DevGrid g;
    long long ps;       // plane stride of the derivative fields
    int zchunk;         // slices per CTA
    int identity_dir;   // direction is the identity: axis-aligned probes
    double probe[3][3]; // index offset of +half a spacing along physical axis d: probe[d][r]
    double isp[3];      // 1 / spacing (the central difference's denominator)
};

// Shared-memory layout (dynamic): input ring [D][HY][HX] float2 (f, m); with a mask, its flags
// [D][HY][HX] bytes; x sums [5][HY][TX] double (+ [HY][TX] int counts); xy-sum ring
// [2R+1][5][TX*TY] double (+ [2R+1][TX*TY] int counts); block-reduction space.
template <int R, int TY, bool MK>
struct Layout {
    static constexpr int HX = TX + 2 * R;
    static constexpr int HY = TY + 2 * R;
    static constexpr int D = R + 2;        // input slices kept: k-R-1 .. k
    static constexpr int W = 2 * R + 1;    // z window
    static constexpr int NT = TX * TY;
    static constexpr int NP = MK ? 4 : 3;  // block partials: cc, |dF|^2, |dM|^2 (+ valid voxels)
    static constexpr size_t in_bytes = sizeof(float2) * D * HY * HX;
    static constexpr size_t vin_bytes = MK ? (size_t)(D * HY * HX + 15) / 16 * 16 : 0;
    static constexpr size_t xs_bytes = sizeof(double) * 5 * HY * TX;
    static constexpr size_t xc_bytes = MK ? sizeof(int) * HY * TX : 0;
    static constexpr size_t ring_bytes = sizeof(double) * W * 5 * NT;
    static constexpr size_t rc_bytes = MK ? sizeof(int) * W * NT : 0;
    static constexpr size_t bytes =
        in_bytes + vin_bytes + xs_bytes + xc_bytes + ring_bytes + rc_bytes + 64 * sizeof(double);
};

// MK: masked (cpu/mod.rs:134-163 -> evaluate_masked with Some(valid)): a voxel counts only where
// `vimg` is not zero; invalid voxels add nothing to any window sum, the count is the number of
// valid voxels in the window, their outputs are zero and the value is the mean over the valid
// voxels (result[3] receives their number; zero means no voxel in the masks).
template <int R, int TY, bool MK>
__global__ void __launch_bounds__(TX * TY) k_cc_pair(CcArgs a, const float* __restrict__ fimg,
                                                     const float* __restrict__ mimg,
                                                     const float* __restrict__ vimg,
                                                     float* __restrict__ d_fixed,
                                                     float* __restrict__ d_moving,
                                                     double* __restrict__ partials,
                                                     unsigned int* __restrict__ counter,
                                                     double* __restrict__ result, int want_norms) {
    using L = Layout<R, TY, MK>;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* in = reinterpret_cast<float2*>(smem);
    unsigned char* vin = smem + L::in_bytes;
    double* xs = reinterpret_cast<double*>(smem + L::in_bytes + L::vin_bytes);
    int* xc = reinterpret_cast<int*>(smem + L::in_bytes + L::vin_bytes + L::xs_bytes);
    double* ring = reinterpret_cast<double*>(smem + L::in_bytes + L::vin_bytes + L::xs_bytes +
                                             L::xc_bytes);
    int* rcn = reinterpret_cast<int*>(ring + L::W * 5 * L::NT);
    double* red = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(rcn) + L::rc_bytes);

    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * a.zchunk;
    const int z1 = min(z0 + a.zchunk, nz);
    const int x = x0 + tx, y = y0 + ty;
    const bool own = x < nx && y < ny;
    const long long sxy = (long long)nx * ny;

    for (int s = tid; s < L::W * 5 * L::NT; s += L::NT) ring[s] = 0.0;
    if constexpr (MK)
        for (int s = tid; s < L::W * L::NT; s += L::NT) rcn[s] = 0;
    double S[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    int Sc = 0;  // valid voxels in the window (masked)
    double acc_cc = 0.0, acc_nf = 0.0, acc_nm = 0.0, acc_nv = 0.0;

    // analytic voxel counts of the clamped window along x and y
    const int cxn = own ? (min(x + R, nx - 1) - max(x - R, 0) + 1) : 0;
    const int cyn = own ? (min(y + R, ny - 1) - max(y - R, 0) + 1) : 0;

    const int kbeg = max(z0 - R, 0);
    const int kend = min(z1 + R, nz);  // slices that exist and are needed (exclusive)
    // slice-invariant prefetch slots: offset inside a slice (-1 outside the image in x or y)
    constexpr int PERC = (L::HY * L::HX + L::NT - 1) / L::NT;
    int src_off[PERC];
#pragma unroll
    for (int q = 0; q < PERC; ++q) {
        int s = tid + q * L::NT;
        src_off[q] = -1;
        if (s < L::HY * L::HX) {
            int hy = s / L::HX, hx = s - hy * L::HX;
            int gx = x0 - R + hx, gy = y0 - R + hy;
            if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) src_off[q] = gy * nx + gx;
        }
    }
    float2 pre[PERC];
    unsigned char prev[PERC];
    auto fetch = [&](int k) {
        const long long zoff = (long long)k * sxy;
#pragma unroll
        for (int q = 0; q < PERC; ++q) {
            pre[q] = src_off[q] >= 0 ? make_float2(__ldg(fimg + zoff + src_off[q]),
                                                   __ldg(mimg + zoff + src_off[q]))
                                     : make_float2(0.0f, 0.0f);
            if constexpr (MK)
                prev[q] = src_off[q] >= 0 ? (__ldg(vimg + zoff + src_off[q]) != 0.0f) : 0;
        }
    };
    if (kbeg < kend) fetch(kbeg);
    for (int k = kbeg; k < z1 + R; ++k) {
        __syncthreads();  // previous slice's readers are done with the slot and the x sums
        double P[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        int Pc = 0;
        const bool have = k < kend;
        if (have) {
            float2* slot = in + (k % L::D) * (L::HY * L::HX);
            unsigned char* vslot = vin + (k % L::D) * (L::HY * L::HX);
#pragma unroll
            for (int q = 0; q < PERC; ++q) {
                int s = tid + q * L::NT;
                if (s < L::HY * L::HX) {
                    slot[s] = pre[q];
                    if constexpr (MK) vslot[s] = prev[q];
                }
            }
            __syncthreads();
            if (k + 1 < kend) fetch(k + 1);  // in flight while this slice is summed
            // x pass: each item makes the sums of two adjacent columns from one window of
            // 2r + 2 voxels (the 2r in the middle are shared)
            for (int s = tid; s < L::HY * (TX / 2); s += L::NT) {
                int hy = s / (TX / 2), cp = s - hy * (TX / 2);
                const float2* row = slot + hy * L::HX + 2 * cp;
                const unsigned char* vrow = vslot + hy * L::HX + 2 * cp;
                // a masked-out voxel enters every sum as zero
                auto val = [&](int t) {
                    float2 v = row[t];
                    if constexpr (MK)
                        if (!vrow[t]) v = make_float2(0.0f, 0.0f);
                    return v;
                };
                if constexpr (MK) {
                    int cn = 0;
#pragma unroll
                    for (int t = 1; t <= 2 * R; ++t) cn += vrow[t];
                    xc[hy * TX + 2 * cp] = cn + vrow[0];
                    xc[hy * TX + 2 * cp + 1] = cn + vrow[2 * R + 1];
                }
                // two interleaved partial sums per plane: half-length add chains
                double c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0;
                double e0 = 0, e1 = 0, e2 = 0, e3 = 0, e4 = 0;
#pragma unroll
                for (int t = 1; t <= 2 * R; t += 2) {
                    float2 v = val(t), w = val(t + 1);
                    double f = v.x, m = v.y, g = w.x, n = w.y;
                    c0 += f;
                    c1 += m;
                    c2 += f * f;
                    c3 += m * m;
                    c4 += f * m;
                    e0 += g;
                    e1 += n;
                    e2 += g * g;
                    e3 += n * n;
                    e4 += g * n;
                }
                c0 += e0;
                c1 += e1;
                c2 += e2;
                c3 += e3;
                c4 += e4;
                float2 va = val(0), vb = val(2 * R + 1);
                double fa = va.x, ma = va.y, fb = vb.x, mb = vb.y;
                double* o = xs + hy * TX + 2 * cp;
                *reinterpret_cast<double2*>(o + 0 * L::HY * TX) = make_double2(c0 + fa, c0 + fb);
                *reinterpret_cast<double2*>(o + 1 * L::HY * TX) = make_double2(c1 + ma, c1 + mb);
                *reinterpret_cast<double2*>(o + 2 * L::HY * TX) = make_double2(c2 + fa * fa, c2 + fb * fb);
                *reinterpret_cast<double2*>(o + 3 * L::HY * TX) = make_double2(c3 + ma * ma, c3 + mb * mb);
                *reinterpret_cast<double2*>(o + 4 * L::HY * TX) = make_double2(c4 + fa * ma, c4 + fb * mb);
            }
            __syncthreads();
            // y pass for the thread's own column
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                double s = 0.0, s2 = 0.0;  // two partial sums: half-length add chains
#pragma unroll
                for (int t = 0; t < 2 * R; t += 2) {
                    s += xs[(q * L::HY + ty + t) * TX + tx];
                    s2 += xs[(q * L::HY + ty + t + 1) * TX + tx];
                }
                P[q] = s + s2 + xs[(q * L::HY + ty + 2 * R) * TX + tx];
            }
            if constexpr (MK) {
#pragma unroll
                for (int t = 0; t <= 2 * R; ++t) Pc += xc[(ty + t) * TX + tx];
            }
        }
        // z window: running sum over the ring of xy sums (entering k, leaving k - 2R - 1)
        double* rs = ring + (k % L::W) * 5 * L::NT + tid;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            double old = rs[q * L::NT];
            S[q] += P[q] - old;
            rs[q * L::NT] = P[q];
        }
        if constexpr (MK) {
            int* rc = rcn + (k % L::W) * L::NT + tid;
            Sc += Pc - *rc;
            *rc = Pc;
        }
        const int z = k - R;
        if (z < z0 || z >= z1 || !own) continue;

        // ---- output voxel (x, y, z) ----
        const long long l = (long long)z * sxy + (long long)y * nx + x;
        double cnt;
        if constexpr (MK) {
            if (!vin[(z % L::D) * (L::HY * L::HX) + (ty + R) * L::HX + (tx + R)]) {
                d_fixed[l] = d_fixed[l + a.ps] = d_fixed[l + 2 * a.ps] = 0.0f;
                d_moving[l] = d_moving[l + a.ps] = d_moving[l + 2 * a.ps] = 0.0f;
                continue;
            }
            cnt = (double)Sc;  // >= 1: the centre is valid
            acc_nv += 1.0;
        } else {
            const int czn = min(z + R, nz - 1) - max(z - R, 0) + 1;
            cnt = (double)(cxn * cyn * czn);
        }
        const float2* cs = in + (z % L::D) * (L::HY * L::HX) + (ty + R) * L::HX + (tx + R);
        const float fv = cs[0].x, mv = cs[0].y;
        // metric/cc.rs:267-302 (same expression order)
        const double sum_f = S[0], sum_m = S[1], sum_f2 = S[2], sum_m2 = S[3], sum_fm = S[4];
        const double icnt = 1.0 / cnt;
        const double fmean = sum_f * icnt, mmean = sum_m * icnt;
        const double s_ff = sum_f2 - fmean * sum_f - fmean * sum_f + cnt * fmean * fmean;
        const double s_mm = sum_m2 - mmean * sum_m - mmean * sum_m + cnt * mmean * mmean;
        const double s_fm = sum_fm - mmean * sum_f - fmean * sum_m + cnt * mmean * fmean;
        const double fi = (double)fv - fmean, mi = (double)mv - mmean;
        const double product = s_ff * s_mm;
        double cc = 1.0, cf = 0.0, cm = 0.0;
        const bool prod_ok = fabs(product) > DBL_EPSILON;
        const bool coef_ok = s_ff > DBL_EPSILON && s_mm > DBL_EPSILON;  // implies product > 0
        // one reciprocal: 1 / sMM = sFF / product and 1 / sFF = sMM / product
        const double ip = (prod_ok || coef_ok) ? 1.0 / product : 0.0;
        if (prod_ok) cc = s_fm * s_fm * ip;
        if (coef_ok) {
            const double k2 = 2.0 * s_fm * ip;
            cf = k2 * (fi - s_fm * s_ff * ip * mi);  // (fixed, moving)
            cm = k2 * (mi - s_fm * s_mm * ip * fi);  // (moving, fixed)
        }
        acc_cc += cc;
        // gradients of moving (for the first direction) and of fixed (for the second)
        float gm[3], gf[3];
        if (a.identity_dir) {
            const int nn[3] = {nx, ny, nz};
            const int pos[3] = {x, y, z};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                gm[d] = 0.0f;
                gf[d] = 0.0f;
                if (!axis_probe_inside(a.g, x, y, z, d, -1.0, nn[d]) ||
                    !axis_probe_inside(a.g, x, y, z, d, +1.0, nn[d]))
                    continue;
                // neighbours along d inside the staged tile / ring
                float2 lo, hi;
                const float2* c0 = cs;
                if (d == 0) {
                    lo = c0[-1];
                    hi = c0[1];
                } else if (d == 1) {
                    lo = c0[-L::HX];
                    hi = c0[L::HX];
                } else {
                    lo = (z > 0) ? in[((z - 1) % L::D) * (L::HY * L::HX) + (ty + R) * L::HX + (tx + R)]
                                 : cs[0];
                    hi = (z < nz - 1) ? in[((z + 1) % L::D) * (L::HY * L::HX) + (ty + R) * L::HX + (tx + R)]
                                      : cs[0];
                }
                const int p = pos[d];
                // upper probe at p + 0.5: lerp to p + 1 unless p is the last voxel
                float m2 = p < nn[d] - 1 ? fmaf(hi.y - mv, 0.5f, mv) : mv;
                float f2 = p < nn[d] - 1 ? fmaf(hi.x - fv, 0.5f, fv) : fv;
                // lower probe at p - 0.5: base p - 1 with weight 0.5, or the first voxel itself
                float m1 = p > 0 ? fmaf(mv - lo.y, 0.5f, lo.y) : mv;
                float f1 = p > 0 ? fmaf(fv - lo.x, 0.5f, lo.x) : fv;
                gm[d] = (float)((double)(m2 - m1) * a.isp[d]);
                gf[d] = (float)((double)(f2 - f1) * a.isp[d]);
            }
        } else {
            central_difference_exact(mimg, a.g, x, y, z, gm);
            central_difference_exact(fimg, a.g, x, y, z, gf);
        }
        const float fcf = (float)cf, fcm = (float)cm;
        float dfx = fcf * gm[0], dfy = fcf * gm[1], dfz = fcf * gm[2];
        float dmx = fcm * gf[0], dmy = fcm * gf[1], dmz = fcm * gf[2];
        d_fixed[l] = dfx;
        d_fixed[l + a.ps] = dfy;
        d_fixed[l + 2 * a.ps] = dfz;
        d_moving[l] = dmx;
        d_moving[l + a.ps] = dmy;
        d_moving[l + 2 * a.ps] = dmz;
        if (want_norms) {
            acc_nf += (double)dfx * dfx + (double)dfy * dfy + (double)dfz * dfz;
            acc_nm += (double)dmx * dmx + (double)dmy * dmy + (double)dmz * dmz;
        }
    }

    // block partials, then the fixed-order last-block reduction
    constexpr int NP = L::NP;
    double acc[4] = {acc_cc, acc_nf, acc_nm, acc_nv};
#pragma unroll
    for (int q = 0; q < NP; ++q) acc[q] = warp_sum_d(acc[q]);
    __syncthreads();
    const int warps = L::NT / 32;
    if ((tid & 31) == 0) {
#pragma unroll
        for (int q = 0; q < NP; ++q) red[(tid >> 5) * NP + q] = acc[q];
    }
    __syncthreads();
    const unsigned int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (tid < NP) {
        double s = 0.0;
        for (int w = 0; w < warps; ++w) s += red[w * NP + tid];
        partials[(size_t)bid * NP + tid] = s;
    }
    __threadfence();
    __syncthreads();
    __shared__ bool last;
    if (tid == 0) last = atomicAdd(counter, 1u) == nblocks - 1;
    __syncthreads();
    if (!last) return;
    if (tid < 32) {
        double tot[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            double s = 0.0;
            for (unsigned int b = tid; b < nblocks; b += 32) s += __ldcg(partials + (size_t)b * NP + q);
            tot[q] = warp_sum_d(s);
        }
        if (tid == 0) {
            // the mean over the valid voxels (all voxels without a mask); no valid voxel: NaN
            result[0] = -tot[0] / (MK ? tot[3] : (double)a.g.n);
            result[1] = tot[1];
            result[2] = tot[2];
            if constexpr (MK) result[3] = tot[3];
            *counter = 0;
        }
    }
}

template <int R, int TY, bool MK>
int launch_r(fw_ctx* ctx, const CcArgs& a0, const float* f, const float* m, const float* v,
             float* df, float* dm, double* d_result, int want_norms) {
    using L = Layout<R, TY, MK>;
    CcArgs a = a0;
    dim3 grid((a.g.nx + TX - 1) / TX, (a.g.ny + TY - 1) / TY, 1);
    // z chunks: enough CTAs to fill the GPU a few times over, chunks no thinner than 4R slices
    long long tiles = (long long)grid.x * grid.y;
    int want = (int)std::max<long long>(1, (4LL * ctx->num_sms + tiles - 1) / tiles);
    int chunk = (a.g.nz + want - 1) / want;
    chunk = std::max(chunk, std::min(a.g.nz, 4 * R + 4));
    a.zchunk = chunk;
    grid.z = (a.g.nz + chunk - 1) / chunk;
    unsigned int nblocks = grid.x * grid.y * grid.z;
    FW_TRY(ensure_scratch(ctx, SLOT_PARTIALS + (size_t)L::NP * nblocks + 16));
    FW_CUDA(cudaFuncSetAttribute(k_cc_pair<R, TY, MK>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes));
    k_cc_pair<R, TY, MK><<<grid, L::NT, L::bytes, ctx->stream>>>(
        a, f, m, v, df, dm, ctx->d_scratch + SLOT_PARTIALS, ctx->d_counter + 1, d_result,
        want_norms);
    return check_launch(ctx, "k_cc_pair");
}

template <bool MK>
int launch_radius(fw_ctx* ctx, const CcArgs& a, int radius, const float* f, const float* m,
                  const float* v, float* df, float* dm, double* d_result, int want_norms) {
    switch (radius) {
        case 1: return launch_r<1, 8, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
        case 2: return launch_r<2, 8, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
        case 3: return launch_r<3, 8, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
        case 4: return launch_r<4, 8, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
        case 5: return launch_r<5, 8, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
        case 6: return launch_r<6, 4, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
        case 7: return launch_r<7, 4, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
        case 8: return launch_r<8, 4, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
        default:
            return fail(FW_ERR_INVALID, "cc metric: radius must be in 1..=8 (BOX_RADIUS_MAX)");
    }
}

}  // namespace

// d_result receives [value, sum |d_fixed|^2, sum |d_moving|^2] and, with `valid`, the number of
// valid voxels in d_result[3].
int launch_cc_pair_impl(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving, int radius,
                        fw_field* d_fixed, fw_field* d_moving, double* d_result, int want_norms,
                        const fw_image* valid) {
    CcArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = dev_grid(fixed->grid);
    a.ps = d_fixed->ps;
    const HostGrid& g = fixed->grid;
    for (int d = 0; d < 3; ++d) a.isp[d] = 1.0 / g.sp[d];
    a.identity_dir = 1;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            if (g.dir[r * 3 + c] != (r == c ? 1.0 : 0.0)) a.identity_dir = 0;
    if (valid)
        return launch_radius<true>(ctx, a, radius, fixed->d, moving->d, valid->d, d_fixed->d,
                                   d_moving->d, d_result, want_norms);
    return launch_radius<false>(ctx, a, radius, fixed->d, moving->d, nullptr, d_fixed->d,
                                d_moving->d, d_result, want_norms);
}

int launch_cc_pair(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving, int radius,
                   fw_field* d_fixed, fw_field* d_moving, double* d_value, double* d_norms) {
    (void)d_norms;
    return launch_cc_pair_impl(ctx, fixed, moving, radius, d_fixed, d_moving, d_value,
                               d_norms != nullptr);
}

}  // namespace fw

using namespace fw;

extern "C" {

static int cc_pair_common(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                          const fw_image* valid, int32_t radius, double values[2],
                          fw_field** d_fixed, fw_field** d_moving, double norms[2]) {
    FW_CHECK(ctx && fixed && moving && values && d_fixed && d_moving, "null argument");
    if (!fixed->grid.same(moving->grid))
        return fail(FW_ERR_INVALID, "cc metric: the images are not on one grid");
    if (valid && !valid->grid.same(fixed->grid))
        return fail(FW_ERR_INVALID, "cc metric: the mask is not on the virtual grid");
    fw_field *a = nullptr, *b = nullptr;
    FW_TRY(new_field(ctx, fixed->grid, &a));
    int rc = new_field(ctx, fixed->grid, &b);
    if (rc) {
        fw_field_free(a);
        return rc;
    }
    // [value, nf, nm, valid voxels] at SLOT_CC_VALUE .. SLOT_CC_VALID
    double* slot = ctx->d_scratch + SLOT_CC_VALUE;
    rc = launch_cc_pair_impl(ctx, fixed, moving, radius, a, b, slot, 1, valid);
    double r[4] = {0, 0, 0, 0};
    if (!rc) rc = read_back(ctx, slot, valid ? 4 : 3, r);
    if (!rc && valid && r[3] == 0.0) rc = fail(FW_ERR_INVALID, std::string("cc metric: ") + FW_NO_VOXEL_IN_MASKS);
    if (rc) {
        fw_field_free(a);
        fw_field_free(b);
        return rc;
    }
    values[0] = r[0];
    values[1] = r[0];
    if (norms) {
        norms[0] = std::sqrt(r[1]);
        norms[1] = std::sqrt(r[2]);
    }
    *d_fixed = a;
    *d_moving = b;
    return 0;
}

int fw_cc_value_derivative_pair(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                                int32_t radius, double values[2], fw_field** d_fixed,
                                fw_field** d_moving) {
    return cc_pair_common(ctx, fixed, moving, nullptr, radius, values, d_fixed, d_moving, nullptr);
}

int fw_cc_value_derivative_pair_with_norms(fw_ctx* ctx, const fw_image* fixed,
                                           const fw_image* moving, int32_t radius,
                                           double values[2], fw_field** d_fixed,
                                           fw_field** d_moving, double norms[2]) {
    FW_CHECK(norms, "null norms");
    return cc_pair_common(ctx, fixed, moving, nullptr, radius, values, d_fixed, d_moving, norms);
}

int fw_cc_value_derivative_pair_masked(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                                       const fw_image* valid, int32_t radius, double values[2],
                                       fw_field** d_fixed, fw_field** d_moving) {
    FW_CHECK(valid, "null mask");
    return cc_pair_common(ctx, fixed, moving, valid, radius, values, d_fixed, d_moving, nullptr);
}

int fw_cc_value_derivative_pair_masked_with_norms(fw_ctx* ctx, const fw_image* fixed,
                                                  const fw_image* moving, const fw_image* valid,
                                                  int32_t radius, double values[2],
                                                  fw_field** d_fixed, fw_field** d_moving,
                                                  double norms[2]) {
    FW_CHECK(valid && norms, "null argument");
    return cc_pair_common(ctx, fixed, moving, valid, radius, values, d_fixed, d_moving, norms);
}

int fw_cc_value_derivative(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                           int32_t radius, double* value, fw_field** derivative) {
    FW_CHECK(value && derivative, "null argument");
    double v[2];
    fw_field *a = nullptr, *b = nullptr;
    FW_TRY(cc_pair_common(ctx, fixed, moving, nullptr, radius, v, &a, &b, nullptr));
    fw_field_free(b);
    *value = v[0];
    *derivative = a;
    return 0;
}

}  // extern "C"

// ---- allocation-free variant of the CC pair ---------------------------------------------------
//
// For callers that cannot allocate device memory: code that records its work inside a CUDA
// stream capture (allocating there breaks the capture), hosts that hand every byte of the GPU to
// their own pool allocator (a deep-learning framework's caching allocator, a serving process
// with a fixed HBM budget) and real-time pipelines that plan all memory before they start. The
// caller passes the images, the two derivative fields and a 3-double result on the device; the
// kernel's only scratch -- the block partials and the last-block counter -- lives in the
// file-scope array below, which every GPU that loads this library holds until the process exits.

namespace fw {
namespace {

struct NoAllocScratch {
    double partials[3 * FW_NOALLOC_MAX_BLOCKS];
    unsigned int counter[64];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_noalloc_mu;
NoAllocScratch* g_noalloc_ptr[128] = {};

// The array's device address on `device` (current), looked up once per device: in host code the
// symbol is only a host-side stand-in, not an address a kernel may use.
int noalloc_scratch(int device, NoAllocScratch** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (device < 0 || device >= 128) return fail(FW_ERR_INVALID, "cc pair (no alloc): device index out of range");
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[device] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_noalloc_ptr[device];
    return 0;
}

template <int R, int TY>
int noalloc_launch(const CcArgs& a0, int num_sms, const float* f, const float* m, float* df,
                   float* dm, double* result, NoAllocScratch* s, cudaStream_t stream) {
    using L = Layout<R, TY, false>;
    CcArgs a = a0;
    dim3 grid((a.g.nx + TX - 1) / TX, (a.g.ny + TY - 1) / TY, 1);
    long long tiles = (long long)grid.x * grid.y;
    int want = (int)std::max<long long>(1, (4LL * num_sms + tiles - 1) / tiles);
    int chunk = (a.g.nz + want - 1) / want;
    chunk = std::max(chunk, std::min(a.g.nz, 4 * R + 4));
    a.zchunk = chunk;
    grid.z = (a.g.nz + chunk - 1) / chunk;
    long long nblocks = (long long)grid.x * grid.y * grid.z;
    if (nblocks > FW_NOALLOC_MAX_BLOCKS)
        return fail(FW_ERR_INVALID,
                    "cc pair (no alloc): the grid needs " + std::to_string(nblocks) +
                        " thread blocks, more than the " + std::to_string(FW_NOALLOC_MAX_BLOCKS) +
                        " the static scratch holds (use fw_cc_value_derivative_pair)");
    // the last-block counter must start at zero whatever the previous call left
    FW_CUDA(cudaMemsetAsync(s->counter, 0, sizeof(unsigned int), stream));
    FW_CUDA(cudaFuncSetAttribute(k_cc_pair<R, TY, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes));
    k_cc_pair<R, TY, false><<<grid, L::NT, L::bytes, stream>>>(a, f, m, nullptr, df, dm,
                                                                s->partials, s->counter, result, 1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k_cc_pair (no alloc)");
    return 0;
}

}  // namespace
}  // namespace fw

extern "C" int fw_cc_value_derivative_pair_noalloc(const fw_grid* grid, const float* fixed,
                                                   const float* moving, int32_t radius,
                                                   float* d_fixed, float* d_moving,
                                                   int64_t plane_stride, double* result,
                                                   void* stream) {
    FW_CHECK(grid && fixed && moving && d_fixed && d_moving && result, "null argument");
    HostGrid g;
    FW_TRY(make_grid(grid, g));
    FW_CHECK(plane_stride >= g.count(), "cc pair (no alloc): plane stride below the voxel count");
    int device = 0;
    FW_CUDA(cudaGetDevice(&device));
    int num_sms = 0;
    FW_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    NoAllocScratch* s = nullptr;
    FW_TRY(noalloc_scratch(device, &s));
    CcArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = dev_grid(g);
    a.ps = plane_stride;
    for (int d = 0; d < 3; ++d) a.isp[d] = 1.0 / g.sp[d];
    a.identity_dir = 1;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            if (g.dir[r * 3 + c] != (r == c ? 1.0 : 0.0)) a.identity_dir = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (radius) {
        case 1: return noalloc_launch<1, 8>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 2: return noalloc_launch<2, 8>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 3: return noalloc_launch<3, 8>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 4: return noalloc_launch<4, 8>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 5: return noalloc_launch<5, 8>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 6: return noalloc_launch<6, 4>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 7: return noalloc_launch<7, 4>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 8: return noalloc_launch<8, 4>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        default:
            return fail(FW_ERR_INVALID, "cc metric: radius must be in 1..=8 (BOX_RADIUS_MAX)");
    }
}
