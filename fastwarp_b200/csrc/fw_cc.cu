// fw_cc.cu -- ANTs neighbourhood cross-correlation, both directions in one pass.
//
// Restates metric/cc.rs:170-321 (CcMetric::evaluate_masked with identity transforms on one grid,
// what cpu/mod.rs:299-331 runs for Backend::cc_value_derivative_pair): the six window sums over a
// clamped (2r+1)^3 box, local CC = sFM^2 / (sFF sMM), value = -mean(localCC), and the derivative
// coefficient * grad(moving) by ITK's half-spacing central difference (interp.rs:96-120).
//
// Kernel design (sm_100a): one CTA owns a TX x TY column tile and marches along z over a chunk
// of slices. The z window comes first, as running sums over the tile's halo columns kept in
// shared memory (entering slice added, leaving slice subtracted); the y and x box passes then run
// on those sums. Sums are float64: products of float32 voxels are exact in float64, so the
// centred second moments (sum f^2 - (sum f)^2 / n) keep their precision in flat bright regions
// where float32 cancels. The window planes never touch HBM: the kernel reads the two images (the
// leaving slice and the halo a second time, from L2) and writes the two derivative fields. Shared
// memory holds the z sums, the y sums and a few raw slices (58 KB at r = 4), and 80 registers a
// thread let three CTAs share an SM and hide each other's float64 and load latency.
#include <cuda_runtime.h>

#include <cfloat>
#include <atomic>
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

// Shared-memory layout (dynamic): the z-window sums of every halo column, [5][HY*HX] double
// (+ [HY*HX] int counts with a mask); y sums [5][HX][TY+1] double, column-major with an odd
// column stride (+ [TY][HX] int counts); the raw voxels of the tile with a one-voxel halo for the
// last D slices, [D][TY+2][TX+2] float2 (f, m), for the centre values and the central
// differences; the x sums of the tile's voxels [5][TX][TY+1] double; block-reduction space.
// The odd strides keep every pass free of bank conflicts: the y pass stores consecutive columns,
// the x pass reads eight rows of two column groups per half-warp, and each voxel's thread reads
// its own row of a column.
template <int R, int TY, bool MK>
struct Layout {
    static constexpr int HX = TX + 2 * R;
    static constexpr int HY = TY + 2 * R;
    static constexpr int HC = HX * HY;           // halo columns of the tile
    static constexpr int NT = TX * TY;
    static constexpr int CPT = (HC + NT - 1) / NT;  // halo columns per thread
    static constexpr int NP = MK ? 4 : 3;  // block partials: cc, |dF|^2, |dM|^2 (+ valid voxels)
    static constexpr int RX = TX + 2, RY = TY + 2, RXY = RX * RY;
    // raw slices kept: the output at step k reads slices k-R-1 .. k-R+1, and slice k is written
    // before step k's first barrier, while slow threads may still read step k-1's outputs
    static constexpr int D = R + 3;
    static constexpr size_t zs1 = sizeof(double) * 5 * HC + (MK ? sizeof(int) * HC : 0);
    static constexpr int YS = TY + 1;                                  // odd: TY is even
    static constexpr int XG = 8;                                       // x outputs per item
    static_assert(TX % XG == 0, "whole x groups");
    static constexpr size_t xs_bytes = sizeof(double) * 5 * HX * YS;  // y sums [5][HX][YS]
    static constexpr size_t xc_bytes = MK ? sizeof(int) * TY * HX : 0;
    static constexpr size_t raw_bytes = sizeof(float2) * D * RXY;
    static constexpr size_t sx_bytes = sizeof(double) * 5 * TX * YS;  // x sums [5][TX][YS]
    static constexpr size_t sx_off = zs1 + xs_bytes + xc_bytes + raw_bytes;
    static constexpr size_t red_off = sx_off + sx_bytes;
    static constexpr size_t bytes = red_off + 64 * sizeof(double);
};

// MK: masked (cpu/mod.rs:134-163 -> evaluate_masked with Some(valid)): a voxel counts only where
// `vimg` is not zero; invalid voxels add nothing to any window sum, the count is the number of
// valid voxels in the window, their outputs are zero and the value is the mean over the valid
// voxels (result[3] receives their number; zero means no voxel in the masks).
//
// Pass order z, y, x. Each thread owns up to CPT halo columns and moves their z-window sums (in
// shared memory, where the y pass reads them) one slice per step: the entering slice is added
// and the leaving slice (read again, from L2) subtracted -- before the step's first barrier, which
// the previous step's y pass has passed. Products of float32 voxels are exact in float64, so the
// running sums carry no drift beyond float64 rounding. The y pass makes column sums of them four
// output rows at a time, the x pass eight outputs of a row at a time, and each thread then reads
// its own voxel's window sums. The kernel is bound by shared-memory bandwidth, which this order spends
// least on: the shared-tap pairs sit in the pass over the wider (halo) extent, and both passes
// read along consecutive banks.
#ifndef FW_CC_MIN_BLOCKS
#define FW_CC_MIN_BLOCKS 3
#endif

// The window sums' arithmetic. SumF64 (the default): float64, in which the products of float32
// voxels are exact. SumC32: compensated float32, a (hi, lo) float pair per sum -- products split
// exactly by an fma (TwoProduct), additions by Knuth's TwoSum with the rounding errors gathered
// in lo and a Fast2Sum renormalisation; every operation is an explicitly rounded intrinsic, so
// the compiler cannot fuse a product into a neighbouring addition. Both take 8 bytes a sum in
// shared memory.
struct SumF64 {
    using T = double;
    __device__ static __forceinline__ T zero() { return 0.0; }
    __device__ static __forceinline__ T diff(float a, float b) { return (double)a - (double)b; }
    __device__ static __forceinline__ T prod_diff(float a, float b, float c, float d) {
        const double x = a, y = b, z = c, w = d;
        return x * y - z * w;
    }
    __device__ static __forceinline__ T add(T a, T b) { return a + b; }
    __device__ static __forceinline__ double value(T a) { return a; }
};

struct SumC32 {
    using T = float2;  // x: hi, y: lo
    __device__ static __forceinline__ void two_sum(float a, float b, float& s, float& e) {
        s = __fadd_rn(a, b);
        const float bb = __fsub_rn(s, a);
        e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    }
    __device__ static __forceinline__ T zero() { return make_float2(0.0f, 0.0f); }
    __device__ static __forceinline__ T diff(float a, float b) {
        float s, e;
        two_sum(a, -b, s, e);
        return make_float2(s, e);
    }
    __device__ static __forceinline__ T prod_diff(float a, float b, float c, float d) {
        const float p = __fmul_rn(a, b), pe = __fmaf_rn(a, b, -p);
        const float q = __fmul_rn(c, d), qe = __fmaf_rn(c, d, -q);
        float s, e;
        two_sum(p, -q, s, e);
        return make_float2(s, __fadd_rn(e, __fsub_rn(pe, qe)));
    }
    __device__ static __forceinline__ T add(T a, T b) {
        float s, e;
        two_sum(a.x, b.x, s, e);
        const float lo = __fadd_rn(e, __fadd_rn(a.y, b.y));
        const float hi = __fadd_rn(s, lo);
        return make_float2(hi, __fsub_rn(lo, __fsub_rn(hi, s)));
    }
    __device__ static __forceinline__ double value(T a) { return (double)a.x + (double)a.y; }
};

// One tile (bx, by, bz) of the CC pair: writes the tile's derivative voxels and leaves the
// thread's sums [cc, |dF|^2, |dM|^2, valid voxels] in acc_out.
template <int R, int TY, bool MK, class Acc = SumF64>
__device__ __forceinline__ void cc_tile(const CcArgs& a, int bx, int by, int bz,
                                        unsigned char* smem, const float* __restrict__ fimg,
                                        const float* __restrict__ mimg,
                                        const float* __restrict__ vimg,
                                        float* __restrict__ d_fixed, float* __restrict__ d_moving,
                                        int want_norms, double acc_out[4]) {
    using L = Layout<R, TY, MK>;
    using T = typename Acc::T;
    static_assert(sizeof(T) == sizeof(double), "a window sum takes 8 bytes");
    T* xs = reinterpret_cast<T*>(smem + L::zs1);
    int* xc = reinterpret_cast<int*>(smem + L::zs1 + L::xs_bytes);
    float2* raw = reinterpret_cast<float2*>(smem + L::zs1 + L::xs_bytes + L::xc_bytes);
    T* sx = reinterpret_cast<T*>(smem + L::sx_off);

    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int x0 = bx * TX, y0 = by * TY;
    const int z0 = bz * a.zchunk;
    const int z1 = min(z0 + a.zchunk, nz);
    const int x = x0 + tx, y = y0 + ty;
    const bool own = x < nx && y < ny;
    const long long sxy = (long long)nx * ny;

    double acc_cc = 0.0, acc_nf = 0.0, acc_nm = 0.0, acc_nv = 0.0;
    // analytic voxel counts of the clamped window along x and y
    const int cxn = own ? (min(x + R, nx - 1) - max(x - R, 0) + 1) : 0;
    const int cyn = own ? (min(y + R, ny - 1) - max(y - R, 0) + 1) : 0;

    // the thread's halo columns: offset inside a slice, -1 outside the image (sums stay zero)
    // and, for columns within one voxel of the tile, their slot in a raw slice (-1 otherwise)
    int coff[L::CPT], ridx[L::CPT];
    T* zs = reinterpret_cast<T*>(smem);
    int* zc = reinterpret_cast<int*>(zs + 5 * L::HC);
#pragma unroll
    for (int j = 0; j < L::CPT; ++j) {
        const int s = tid + j * L::NT;
        coff[j] = -1;
        ridx[j] = -1;
        if (s < L::HC) {
            const int hy = s / L::HX, hx = s - hy * L::HX;
            const int gx = x0 - R + hx, gy = y0 - R + hy;
            if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) coff[j] = gy * nx + gx;
            const int rx = hx - (R - 1), ry = hy - (R - 1);
            if (rx >= 0 && rx < L::RX && ry >= 0 && ry < L::RY) ridx[j] = ry * L::RX + rx;
        }
        if (s < L::HC) {
#pragma unroll
            for (int q = 0; q < 5; ++q) zs[q * L::HC + s] = Acc::zero();
            if constexpr (MK) zc[s] = 0;
        }
    }
    // Non-zero voxels of each halo column's z window, fixed in the low byte, moving in the next
    // (exact integers, never negative). The reference forms every window sum directly from the
    // window's voxels (metric/cc.rs:137-157), so a window where an image is zero sums to exactly
    // zero and its CC takes the degenerate value; a running sum keeps a float64 rounding residue
    // of what entered and left, so the sums of an image are reset to zero whenever its count is.
    int nzc[L::CPT];
#pragma unroll
    for (int j = 0; j < L::CPT; ++j) nzc[j] = 0;
    // entering slice k and leaving slice k - 2R - 1 of the next step, in flight during a step
    float2 pin[L::CPT], pout[L::CPT];
    bool vin[L::CPT], vout[L::CPT];
    const int kb = max(z0 - R, 0);
    auto fetch = [&](int k) {
        const bool add = k < nz, sub = k - 2 * R - 1 >= kb;
        const long long zi = (long long)k * sxy, zo = (long long)(k - 2 * R - 1) * sxy;
#pragma unroll
        for (int j = 0; j < L::CPT; ++j) {
            const bool c = coff[j] >= 0;
            pin[j] = c && add ? make_float2(__ldg(fimg + zi + coff[j]), __ldg(mimg + zi + coff[j]))
                              : make_float2(0.0f, 0.0f);
            pout[j] = c && sub ? make_float2(__ldg(fimg + zo + coff[j]), __ldg(mimg + zo + coff[j]))
                               : make_float2(0.0f, 0.0f);
            if constexpr (MK) {  // pin stays raw: the central differences read it
                vin[j] = c && add && __ldg(vimg + zi + coff[j]) != 0.0f;
                vout[j] = c && sub && __ldg(vimg + zo + coff[j]) != 0.0f;
                if (!vout[j]) pout[j] = make_float2(0.0f, 0.0f);
            }
        }
    };
    fetch(kb);
    for (int k = kb; k < z1 + R; ++k) {
        // z step: add slice k (if it exists), drop slice k - 2R - 1 (if it was added)
        float2* rslot = raw + (k % L::D) * L::RXY;
#pragma unroll
        for (int j = 0; j < L::CPT; ++j) {
            if (ridx[j] >= 0 && k < nz) rslot[ridx[j]] = pin[j];
            float2 a = pin[j];
            if constexpr (MK)
                if (!vin[j]) a = make_float2(0.0f, 0.0f);  // a masked-out voxel adds nothing
            const float f = a.x, m = a.y, g = pout[j].x, n = pout[j].y;
            const int s = tid + j * L::NT;
            if (s < L::HC) {
                T* zq = zs + s;
                nzc[j] += ((int)(f != 0.0f) - (int)(g != 0.0f)) +
                          256 * ((int)(m != 0.0f) - (int)(n != 0.0f));
                const bool fz = (nzc[j] & 255) == 0, mz = (nzc[j] >> 8) == 0;
                zq[0] = fz ? Acc::zero() : Acc::add(zq[0], Acc::diff(f, g));
                zq[L::HC] = mz ? Acc::zero() : Acc::add(zq[L::HC], Acc::diff(m, n));
                zq[2 * L::HC] = fz ? Acc::zero() : Acc::add(zq[2 * L::HC], Acc::prod_diff(f, f, g, g));
                zq[3 * L::HC] = mz ? Acc::zero() : Acc::add(zq[3 * L::HC], Acc::prod_diff(m, m, n, n));
                zq[4 * L::HC] = (fz || mz) ? Acc::zero()
                                           : Acc::add(zq[4 * L::HC], Acc::prod_diff(f, m, g, n));
                if constexpr (MK) zc[s] += (int)vin[j] - (int)vout[j];
            }
        }
        if (k + 1 < z1 + R) fetch(k + 1);
        const int z = k - R;
        if (z < z0) continue;  // the window is still filling (uniform across the CTA)

        __syncthreads();  // z sums visible; the previous x pass is done with the y sums
        // y pass: each item makes four output rows of one halo column for one of the five window
        // sums from one window of 2r + 4 rows, as two pairs of adjacent rows whose 2r middle rows are
        // shared (each pair's sums in the same order as alone); a warp's items are consecutive
        // columns, so its loads and stores fall on distinct banks
        static_assert(TY % 4 == 0, "the y pass makes output rows in fours");
        for (int s = tid; s < 5 * L::HX * (TY / 4); s += L::NT) {
            const int q = s / (L::HX * (TY / 4)), rr = s - q * (L::HX * (TY / 4));
            const int rq = rr / L::HX, hx = rr - rq * L::HX;
            const T* col = zs + q * L::HC + 4 * rq * L::HX + hx;
            T v[2 * R + 4];
#pragma unroll
            for (int t = 0; t < 2 * R + 4; ++t) v[t] = col[t * L::HX];
            T* o = xs + (q * L::HX + hx) * L::YS + 4 * rq;
#pragma unroll
            for (int p2 = 0; p2 < 4; p2 += 2) {
                T c = Acc::zero(), e = Acc::zero();  // two partial sums: half-length add chains
#pragma unroll
                for (int t = 1; t <= 2 * R; t += 2) {
                    c = Acc::add(c, v[p2 + t]);
                    e = Acc::add(e, v[p2 + t + 1]);
                }
                c = Acc::add(c, e);
                o[p2] = Acc::add(c, v[p2]);
                o[p2 + 1] = Acc::add(c, v[p2 + 2 * R + 1]);
            }
            if constexpr (MK) {
                if (q == 0) {
                    const int* ccol = zc + 4 * rq * L::HX + hx;
#pragma unroll
                    for (int p2 = 0; p2 < 4; p2 += 2) {
                        int cn = 0;
#pragma unroll
                        for (int t = 1; t <= 2 * R; ++t) cn += ccol[(p2 + t) * L::HX];
                        xc[(4 * rq + p2) * L::HX + hx] = cn + ccol[p2 * L::HX];
                        xc[(4 * rq + p2 + 1) * L::HX + hx] = cn + ccol[(p2 + 2 * R + 1) * L::HX];
                    }
                }
            }
        }
        __syncthreads();
        // x pass: each item makes the sums of XG consecutive outputs of one row from one window
        // of XG + 2r columns (each output's sum in the same order as alone: even taps, odd taps,
        // the last); a half-warp's items are eight rows of two column groups
        for (int s = tid; s < 5 * TY * (TX / L::XG); s += L::NT) {
            const int q = s / (TY * (TX / L::XG)), rr = s - q * (TY * (TX / L::XG));
            const int row = rr % TY, g = rr / TY;
            const T* in = xs + (q * L::HX + g * L::XG) * L::YS + row;
            T v[L::XG + 2 * R];
#pragma unroll
            for (int t = 0; t < L::XG + 2 * R; ++t) v[t] = in[t * L::YS];
            T* out = sx + (q * TX + g * L::XG) * L::YS + row;
#pragma unroll
            for (int j = 0; j < L::XG; ++j) {
                T e = Acc::zero(), o = Acc::zero();
#pragma unroll
                for (int t = 0; t < 2 * R; t += 2) {
                    e = Acc::add(e, v[j + t]);
                    o = Acc::add(o, v[j + t + 1]);
                }
                out[j * L::YS] = Acc::add(Acc::add(e, o), v[j + 2 * R]);
            }
        }
        __syncthreads();
        if (!own) continue;
        double S[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) S[q] = Acc::value(sx[(q * TX + tx) * L::YS + ty]);

        // ---- output voxel (x, y, z) ----
        const long long l = (long long)z * sxy + (long long)y * nx + x;
        double cnt;
        if constexpr (MK) {
            if (__ldg(vimg + l) == 0.0f) {
                d_fixed[l] = d_fixed[l + a.ps] = d_fixed[l + 2 * a.ps] = 0.0f;
                d_moving[l] = d_moving[l + a.ps] = d_moving[l + 2 * a.ps] = 0.0f;
                continue;
            }
            int Sc = 0;
#pragma unroll
            for (int t = 0; t <= 2 * R; ++t) Sc += xc[ty * L::HX + tx + t];
            cnt = (double)Sc;  // >= 1: the centre is valid
            acc_nv += 1.0;
        } else {
            const int czn = min(z + R, nz - 1) - max(z - R, 0) + 1;
            cnt = (double)(cxn * cyn * czn);
        }
        const float2* cs = raw + (z % L::D) * L::RXY + (ty + 1) * L::RX + (tx + 1);
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
            // interp.rs:96-120 on an identity-direction grid: the probes at +-half a spacing lerp
            // halfway toward the neighbours along the axis, read from the raw slices
            const int nn[3] = {nx, ny, nz};
            const int pos[3] = {x, y, z};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                gm[d] = 0.0f;
                gf[d] = 0.0f;
                if (!axis_probe_inside(a.g, x, y, z, d, -1.0, nn[d]) ||
                    !axis_probe_inside(a.g, x, y, z, d, +1.0, nn[d]))
                    continue;
                const int p = pos[d];
                float2 lo = cs[0], hi = cs[0];
                if (d == 0) {
                    if (p > 0) lo = cs[-1];
                    if (p < nn[d] - 1) hi = cs[1];
                } else if (d == 1) {
                    if (p > 0) lo = cs[-L::RX];
                    if (p < nn[d] - 1) hi = cs[L::RX];
                } else {
                    const int o = (ty + 1) * L::RX + (tx + 1);
                    if (p > 0) lo = raw[((z - 1) % L::D) * L::RXY + o];
                    if (p < nn[d] - 1) hi = raw[((z + 1) % L::D) * L::RXY + o];
                }
                // upper probe at p + 0.5: lerp to p + 1 unless p is the last voxel; lower probe
                // at p - 0.5: base p - 1 with weight 0.5, or the first voxel itself
                const float m2 = p < nn[d] - 1 ? fmaf(hi.y - mv, 0.5f, mv) : mv;
                const float f2 = p < nn[d] - 1 ? fmaf(hi.x - fv, 0.5f, fv) : fv;
                const float m1 = p > 0 ? fmaf(mv - lo.y, 0.5f, lo.y) : mv;
                const float f1 = p > 0 ? fmaf(fv - lo.x, 0.5f, lo.x) : fv;
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

    acc_out[0] = acc_cc;
    acc_out[1] = acc_nf;
    acc_out[2] = acc_nm;
    acc_out[3] = acc_nv;
}

// The block's sums of acc (NP of them) into dst[0 .. NP) (warp sums, then warps in order).
template <int NP, int NT>
__device__ __forceinline__ void cc_block_partials(double acc[4], double* red, double* dst) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < NP; ++q) acc[q] = warp_sum_d(acc[q]);
    __syncthreads();
    if ((tid & 31) == 0) {
#pragma unroll
        for (int q = 0; q < NP; ++q) red[(tid >> 5) * NP + q] = acc[q];
    }
    __syncthreads();
    if (tid < NP) {
        double s = 0.0;
        for (int w = 0; w < NT / 32; ++w) s += red[w * NP + tid];
        dst[tid] = s;
    }
}

// Whether this block is the last of `total` to add its partials (fixed-order reduction).
__device__ __forceinline__ bool cc_last(unsigned int* counter, unsigned int total) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == total - 1;
    __syncthreads();
    return last;
}

// The last block's reduction of `nblocks` partials in a fixed order (every thread of the block,
// block_sum_fixed): [value, |dF|^2, |dM|^2 (, valid voxels)] into result; the counter is reset.
// `red` is the block's shared reduction space (NT / 32 doubles at least).
template <int NP, bool MK>
__device__ __forceinline__ void cc_finish(const double* partials, unsigned int nblocks,
                                          long long n, double* result, unsigned int* counter,
                                          double* red) {
    double tot[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < NP; ++q) tot[q] = block_sum_fixed(partials + q, nblocks, NP, red);
    if (threadIdx.x == 0) {
        // the mean over the valid voxels (all voxels without a mask); no valid voxel: NaN
        result[0] = -tot[0] / (MK ? tot[3] : (double)n);
        result[1] = tot[1];
        result[2] = tot[2];
        if constexpr (MK) result[3] = tot[3];
        *counter = 0;
    }
}

template <int R, int TY, bool MK, class Acc = SumF64>
__global__ void __launch_bounds__(TX * TY, FW_CC_MIN_BLOCKS) k_cc_pair(CcArgs a, const float* __restrict__ fimg,
                                                     const float* __restrict__ mimg,
                                                     const float* __restrict__ vimg,
                                                     float* __restrict__ d_fixed,
                                                     float* __restrict__ d_moving,
                                                     double* __restrict__ partials,
                                                     unsigned int* __restrict__ counter,
                                                     double* __restrict__ result, int want_norms) {
    pdl_wait();
    using L = Layout<R, TY, MK>;
    extern __shared__ __align__(16) unsigned char smem[];
    double* red = reinterpret_cast<double*>(smem + L::red_off);
    double acc[4];
    cc_tile<R, TY, MK, Acc>(a, blockIdx.x, blockIdx.y, blockIdx.z, smem, fimg, mimg, vimg,
                            d_fixed, d_moving, want_norms, acc);
    // block partials, then the fixed-order last-block reduction
    const unsigned int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    cc_block_partials<L::NP, L::NT>(acc, red, partials + (size_t)bid * L::NP);
    if (!cc_last(counter, nblocks)) return;
    cc_finish<L::NP, MK>(partials, nblocks, a.g.n, result, counter, red);
}

// The CC pair of every active subject of a batch (unmasked): subject b's images at
// fimg / mimg + b * img_stride, its derivative fields at d_fixed / d_moving + b * field_stride,
// its tile partials at partials + b * part_stride, its last-tile counter at counter[b] and its
// [value, |dF|^2, |dM|^2] at result + b * result_stride. Tiles are summed in the single
// kernel's block order, so a subject's value does not depend on the batch.
template <int R, int TY>
__global__ void __launch_bounds__(TX * TY, FW_CC_MIN_BLOCKS) k_cc_pair_batch(
    CcArgs a, BatchList Lb, const float* __restrict__ fimg, const float* __restrict__ mimg,
    long long img_stride, float* __restrict__ d_fixed, float* __restrict__ d_moving,
    long long field_stride, double* __restrict__ partials, long long part_stride,
    unsigned int* __restrict__ counter, double* __restrict__ result, int result_stride,
    int want_norms) {
    using L = Layout<R, TY, false>;
    extern __shared__ __align__(16) unsigned char smem[];
    double* red = reinterpret_cast<double*>(smem + L::red_off);
    const int work = *Lb.count * Lb.tiles;
    const int gx = (a.g.nx + TX - 1) / TX, gy = (a.g.ny + TY - 1) / TY;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = Lb.active[w / Lb.tiles], t = w % Lb.tiles;
        int bx, by, bz;
        tile_coords(t, gx, gy, bx, by, bz);
        double acc[4];
        cc_tile<R, TY, false>(a, bx, by, bz, smem, fimg + b * img_stride, mimg + b * img_stride,
                              nullptr, d_fixed + b * field_stride, d_moving + b * field_stride,
                              want_norms, acc);
        double* pb = partials + b * part_stride;
        cc_block_partials<L::NP, L::NT>(acc, red, pb + (size_t)t * L::NP);
        if (cc_last(counter + b, (unsigned int)Lb.tiles))
            cc_finish<L::NP, false>(pb, (unsigned int)Lb.tiles, a.g.n,
                                    result + (size_t)b * result_stride, counter + b, red);
        __syncthreads();  // the next tile rewrites the shared sums
    }
}

// Grid of a launch: TX x TY column tiles times z chunks. About three and a half waves of resident
// CTAs (measured at the 193 x 229 x 193 finest level, r = 4: 8 chunks 0.398 ms, 5 chunks 0.401 ms,
// 2 chunks -- less than one wave -- 0.426 ms), with chunks no thinner than 2R slices, the filling
// steps every chunk pays before its first output.
template <int R, int TY, bool MK, class Acc = SumF64>
int plan_launch(CcArgs& a, int num_sms, dim3* grid) {
    using L = Layout<R, TY, MK>;
    FW_CUDA(cudaFuncSetAttribute(k_cc_pair<R, TY, MK, Acc>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes));
    static const int occ = [] {
        int o = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_cc_pair<R, TY, MK, Acc>, L::NT,
                                                          L::bytes) != cudaSuccess || o < 1)
            o = 1;
        return o;
    }();
    dim3 g((a.g.nx + TX - 1) / TX, (a.g.ny + TY - 1) / TY, 1);
    const long long tiles = (long long)g.x * g.y;
    const long long slots = (long long)occ * num_sms;
    long long best = (7 * slots + tiles) / (2 * tiles);  // round(3.5 slots / tiles)
    best = std::min<long long>(best, a.g.nz / (2 * R));
    best = std::max<long long>(best, 1);
    a.zchunk = (int)((a.g.nz + best - 1) / best);
    g.z = (a.g.nz + a.zchunk - 1) / a.zchunk;
    *grid = g;
    return 0;
}

template <int R, int TY, bool MK, class Acc = SumF64>
int launch_r(fw_ctx* ctx, const CcArgs& a0, const float* f, const float* m, const float* v,
             float* df, float* dm, double* d_result, int want_norms) {
    using L = Layout<R, TY, MK>;
    CcArgs a = a0;
    dim3 grid;
    FW_TRY((plan_launch<R, TY, MK, Acc>(a, ctx->num_sms, &grid)));
    unsigned int nblocks = grid.x * grid.y * grid.z;
    FW_TRY(ensure_scratch(ctx, SLOT_PARTIALS + (size_t)L::NP * nblocks + 16));
    return launch_pdl(ctx, "k_cc_pair", k_cc_pair<R, TY, MK, Acc>, grid, dim3(L::NT), L::bytes,
                      a, f, m, v, df, dm, ctx->d_scratch + SLOT_PARTIALS, ctx->d_counter + 1,
                      d_result, want_norms);
}

// The window-sum arithmetic of the unmasked single-image CC pair (FW_CC_SUMS_*), process-wide.
std::atomic<int> g_cc_sums{FW_CC_SUMS_F64};

template <bool MK>
int launch_radius(fw_ctx* ctx, const CcArgs& a, int radius, const float* f, const float* m,
                  const float* v, float* df, float* dm, double* d_result, int want_norms) {
    const bool c32 = !MK && g_cc_sums.load() == FW_CC_SUMS_C32;
#define FW_CC_RADIUS(RR)                                                                         \
    case RR:                                                                                    \
        if constexpr (!MK)                                                                      \
            if (c32) return launch_r<RR, 8, false, SumC32>(ctx, a, f, m, v, df, dm, d_result,   \
                                                          want_norms);                          \
        return launch_r<RR, 8, MK>(ctx, a, f, m, v, df, dm, d_result, want_norms);
    switch (radius) {
        FW_CC_RADIUS(1)
        FW_CC_RADIUS(2)
        FW_CC_RADIUS(3)
        FW_CC_RADIUS(4)
        FW_CC_RADIUS(5)
        FW_CC_RADIUS(6)
        FW_CC_RADIUS(7)
        FW_CC_RADIUS(8)
        default:
            return fail(FW_ERR_INVALID, "cc metric: radius must be in 1..=8 (BOX_RADIUS_MAX)");
    }
#undef FW_CC_RADIUS
}

template <int R>
int launch_cc_batch_r(fw_ctx* ctx, const CcArgs& a, const BatchList& L, int blocks,
                      const float* f, const float* m, long long img_stride, float* df, float* dm,
                      long long field_stride, double* partials, long long part_stride,
                      unsigned int* counter, double* result, int result_stride, int want_norms) {
    using Lay = Layout<R, 8, false>;
    FW_CUDA(cudaFuncSetAttribute(k_cc_pair_batch<R, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Lay::bytes));
    k_cc_pair_batch<R, 8><<<blocks, Lay::NT, Lay::bytes, ctx->stream>>>(
        a, L, f, m, img_stride, df, dm, field_stride, partials, part_stride, counter, result,
        result_stride, want_norms);
    return check_launch(ctx, "k_cc_pair_batch");
}

template <int R>
int cc_batch_occupancy() {
    using Lay = Layout<R, 8, false>;
    cudaFuncSetAttribute(k_cc_pair_batch<R, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Lay::bytes);
    int o = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_cc_pair_batch<R, 8>, Lay::NT,
                                                      Lay::bytes) != cudaSuccess || o < 1) {
        cudaGetLastError();
        o = 1;
    }
    return o;
}

CcArgs cc_args(const HostGrid& g, long long ps) {
    CcArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = dev_grid(g);
    a.ps = ps;
    for (int d = 0; d < 3; ++d) a.isp[d] = 1.0 / g.sp[d];
    a.identity_dir = 1;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            if (g.dir[r * 3 + c] != (r == c ? 1.0 : 0.0)) a.identity_dir = 0;
    return a;
}

}  // namespace

int cc_batch_tiles(const HostGrid& g, int zchunk) {
    const long long gx = (g.n[0] + TX - 1) / TX, gy = (g.n[1] + 7) / 8;
    const long long gz = (g.n[2] + zchunk - 1) / zchunk;
    return (int)(gx * gy * gz);
}

int cc_batch_blocks_per_sm(int radius) {
    switch (radius) {
        case 1: return cc_batch_occupancy<1>();
        case 2: return cc_batch_occupancy<2>();
        case 3: return cc_batch_occupancy<3>();
        case 4: return cc_batch_occupancy<4>();
        case 5: return cc_batch_occupancy<5>();
        case 6: return cc_batch_occupancy<6>();
        case 7: return cc_batch_occupancy<7>();
        case 8: return cc_batch_occupancy<8>();
        default: return 1;
    }
}

int launch_cc_pair_batch(fw_ctx* ctx, const HostGrid& g, long long ps, int radius, int zchunk,
                         const BatchList& L, int blocks, const float* fimg, const float* mimg,
                         long long img_stride, float* d_fixed, float* d_moving,
                         long long field_stride, double* partials, long long part_stride,
                         unsigned int* counter, double* result, int result_stride,
                         int want_norms) {
    CcArgs a = cc_args(g, ps);
    a.zchunk = zchunk;
#define FW_CC_BATCH(RR)                                                                          \
    case RR:                                                                                    \
        return launch_cc_batch_r<RR>(ctx, a, L, blocks, fimg, mimg, img_stride, d_fixed,         \
                                     d_moving, field_stride, partials, part_stride, counter,     \
                                     result, result_stride, want_norms);
    switch (radius) {
        FW_CC_BATCH(1)
        FW_CC_BATCH(2)
        FW_CC_BATCH(3)
        FW_CC_BATCH(4)
        FW_CC_BATCH(5)
        FW_CC_BATCH(6)
        FW_CC_BATCH(7)
        FW_CC_BATCH(8)
        default:
            return fail(FW_ERR_INVALID, "cc metric: radius must be in 1..=8 (BOX_RADIUS_MAX)");
    }
#undef FW_CC_BATCH
}

// d_result receives [value, sum |d_fixed|^2, sum |d_moving|^2] and, with `valid`, the number of
// valid voxels in d_result[3].
int launch_cc_pair_impl(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving, int radius,
                        fw_field* d_fixed, fw_field* d_moving, double* d_result, int want_norms,
                        const fw_image* valid) {
    CcArgs a = cc_args(fixed->grid, d_fixed->ps);
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

int fw_set_cc_window_sums(int32_t kind) {
    FW_CHECK(kind == FW_CC_SUMS_F64 || kind == FW_CC_SUMS_C32,
             "cc metric: unknown window-sum arithmetic");
    g_cc_sums.store(kind);
    return 0;
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
// For callers that cannot allocate device memory: hosts that hand every byte of the GPU to
// their own pool allocator (a deep-learning framework's caching allocator, a serving process
// with a fixed HBM budget), plug-ins that get only the buffers such a host gives them, and
// real-time pipelines that plan all memory before they start. The
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
    dim3 grid;
    FW_TRY((plan_launch<R, TY, false>(a, num_sms, &grid)));
    long long nblocks = (long long)grid.x * grid.y * grid.z;
    if (nblocks > FW_NOALLOC_MAX_BLOCKS)
        return fail(FW_ERR_INVALID,
                    "cc pair (no alloc): the grid needs " + std::to_string(nblocks) +
                        " thread blocks, more than the " + std::to_string(FW_NOALLOC_MAX_BLOCKS) +
                        " the static scratch holds (use fw_cc_value_derivative_pair)");
    // the last-block counter must start at zero whatever the previous call left
    FW_CUDA(cudaMemsetAsync(s->counter, 0, sizeof(unsigned int), stream));
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
        case 6: return noalloc_launch<6, 8>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 7: return noalloc_launch<7, 8>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        case 8: return noalloc_launch<8, 8>(a, num_sms, fixed, moving, d_fixed, d_moving, result, s, st);
        default:
            return fail(FW_ERR_INVALID, "cc metric: radius must be in 1..=8 (BOX_RADIUS_MAX)");
    }
}
