// fw_smooth.cu -- SyN's Gaussian smoothing of a displacement field (field_ops.rs:478-574) with
// the max |u/sp| reduction of ScaleUpdateField fused into its epilogue (field_ops.rs:191-203),
// and the recursive (Deriche) Gaussian of the level pyramid (pyramid.rs:186-427) on the device.
//
// Gaussian kernel design: one CTA owns a TX x TY column tile and marches along z. Each input
// slice (edge-replicated halo in x and y) is staged in shared memory; the x and y passes run
// there and every xy-smoothed slice enters a ring of 2r+1 slices from which the z pass of the
// output slice is taken. The three components are processed together; one HBM read and one
// HBM write per component.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>
#include <vector>

#include "fw_internal.cuh"

namespace fw {

// field_ops.rs:394-476 -- ITK GaussianOperator's modified Bessel functions (Abramowitz & Stegun
// 9.8.1-4 polynomial fits for I0 and I1, Miller's downward recurrence for I_n).
static double bessel_i0(double y) {
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

static double bessel_i1(double y) {
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

static double bessel_in(int n, double y) {
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

namespace {

constexpr int STX = 32;
constexpr int STY = 8;
constexpr int SNT = STX * STY;
constexpr int MAX_TAPS = 2 * 24 + 1;  // radius <= 24

struct SmoothArgs {
    DevGrid g;
    long long ps_in, ps_out;
    int rx, ry, rz;
    int zchunk;
    float w1, w2;  // blend of smoothed and original (field_ops.rs:546-550)
    float tx_[MAX_TAPS], ty_[MAX_TAPS], tz_[MAX_TAPS];
};

__global__ void __launch_bounds__(SNT) k_smooth(SmoothArgs a, const float* __restrict__ in,
                                                float* __restrict__ out,
                                                unsigned int* __restrict__ max_bits) {
    extern __shared__ __align__(16) float sm[];
    const int HX = STX + 2 * a.rx, HY = STY + 2 * a.ry, W = 2 * a.rz + 1;
    float* tile = sm;                       // [3][HY][HX]
    float* xs = tile + 3 * HY * HX;         // [3][HY][STX]
    float* ring = xs + 3 * HY * STX;        // [W][3][SNT]
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int tid = threadIdx.x, tx = tid % STX, ty = tid / STX;
    const int x0 = blockIdx.x * STX, y0 = blockIdx.y * STY;
    const int z0 = blockIdx.z * a.zchunk, z1 = min(z0 + a.zchunk, nz);
    const int x = x0 + tx, y = y0 + ty;
    const bool own = x < nx && y < ny;
    const long long sxy = (long long)nx * ny;
    float vmax = 0.0f;
    const float isx = (float)(1.0 / a.g.sp[0]), isy = (float)(1.0 / a.g.sp[1]),
                isz = (float)(1.0 / a.g.sp[2]);
    for (int k = z0 - a.rz; k < z1 + a.rz; ++k) {
        __syncthreads();
        const int kz = min(max(k, 0), nz - 1);  // edge replication along z
        const long long zoff = (long long)kz * sxy;
        for (int s = tid; s < HY * HX; s += SNT) {
            int hy = s / HX, hx = s - hy * HX;
            int gx = min(max(x0 - a.rx + hx, 0), nx - 1);
            int gy = min(max(y0 - a.ry + hy, 0), ny - 1);
            long long o = zoff + (long long)gy * nx + gx;
            tile[s] = __ldg(in + o);
            tile[HY * HX + s] = __ldg(in + o + a.ps_in);
            tile[2 * HY * HX + s] = __ldg(in + o + 2 * a.ps_in);
        }
        __syncthreads();
        for (int s = tid; s < HY * STX; s += SNT) {
            int hy = s / STX, cx = s - hy * STX;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float* row = tile + c * HY * HX + hy * HX + cx;
                float acc = 0.0f;
                for (int t = 0; t <= 2 * a.rx; ++t) acc = fmaf(a.tx_[t], row[t], acc);
                xs[c * HY * STX + s] = acc;
            }
        }
        __syncthreads();
        float* rs = ring + ((k - (z0 - a.rz)) % W) * 3 * SNT + tid;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float acc = 0.0f;
            for (int t = 0; t <= 2 * a.ry; ++t)
                acc = fmaf(a.ty_[t], xs[c * HY * STX + (ty + t) * STX + tx], acc);
            rs[c * SNT] = acc;
        }
        const int z = k - a.rz;
        if (z < z0 || !own) continue;
        // z pass over the ring: slices z - rz .. z + rz (virtual indices, replicated at the ends)
        float v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float acc = 0.0f;
            for (int t = 0; t <= 2 * a.rz; ++t) {
                int kk = z - a.rz + t;
                acc = fmaf(a.tz_[t], ring[((kk - (z0 - a.rz)) % W) * 3 * SNT + c * SNT + tid], acc);
            }
            v[c] = acc;
        }
        const long long l = (long long)z * sxy + (long long)y * nx + x;
        const bool face = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
        float o[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float orig = a.w2 != 0.0f ? __ldg(in + l + c * a.ps_in) : 0.0f;
            o[c] = face ? 0.0f : (a.w2 != 0.0f ? v[c] * a.w1 + orig * a.w2 : v[c]);
            out[l + c * a.ps_out] = o[c];
        }
        if (max_bits) {
            float px = o[0] * isx, py = o[1] * isy, pz = o[2] * isz;
            vmax = __int_as_float(max(__float_as_int(vmax),
                                      __float_as_int(nan_canon(sqrtf(px * px + py * py + pz * pz)))));
        }
    }
    if (max_bits) {
        vmax = warp_max_f(vmax);
        if ((tid & 31) == 0 && vmax > 0.0f) atomicMax(max_bits, __float_as_uint(vmax));
    }
}

// ---- fixed-radius path (the same taps on the three axes, the usual case) ----------------------
//
// The separable filter as two bandwidth-bound sweeps instead of one fused 2.5D kernel (whose z
// ring of registers shifts every slice and whose x pass repeats the y halo rows): k_smooth_xy
// filters each z slice along x then y through shared memory (32 x 32 output tile, clamped halo)
// into a temporary field; k_smooth_z filters along z from a fixed-index register window of
// Z_SEG + 2R values per column and applies the faces, the w1/w2 blend and the fused max norm.
// Both passes accumulate taps in the reference's order (field_ops.rs:508-528), x then y then z.

constexpr int XY_T = 32;     // output tile edge of the xy pass
constexpr int XY_NT = 256;   // threads: 32 columns x 8 rows, 4 output rows each
constexpr int Z_SEG = 16;    // z outputs per thread of the z pass

// One 32 x 32 tile (bx, by) of slice z of the xy pass.
template <int R>
__device__ __forceinline__ void smooth_xy_tile(const SmoothArgs& a, int bx, int by, int z,
                                               float* smem_xy, const float* __restrict__ in,
                                               float* __restrict__ tmp, long long ps_tmp) {
    constexpr int HX = XY_T + 2 * R, HY = XY_T + 2 * R;
    constexpr int HXP = (HX + 3) & ~3;       // rows start on 16 bytes
    constexpr int NV = (4 + 2 * R + 3) / 4;  // float4 loads per x window of four outputs
    constexpr int TILE = HY * HXP;
    // the three components' tiles at once (dynamic: [3][TILE] + pad, then [3][HY][32] x sums):
    // all their loads in flight together, two barriers per block
    float* tile = smem_xy;
    float* xs = smem_xy + 3 * TILE + 4 * NV;
    const int nx = a.g.nx, ny = a.g.ny;
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    const int x0 = bx * XY_T, y0 = by * XY_T;
    const long long zoff = (long long)z * nx * ny;
    const int x = x0 + tx;
    static_assert(HX <= 64, "a lane loads two halo columns");
    {
        // halo rows by warps: lane l loads halo columns l and l + 32 (edge replication)
        const int warp = tid >> 5;
        const int gxa = min(max(x0 - R + tx, 0), nx - 1);
        const int gxb = min(max(x0 - R + tx + 32, 0), nx - 1);
        const bool second = tx + 32 < HX;
        const float* plane = in + zoff;
        for (int hy = warp; hy < HY; hy += XY_NT / 32) {
            const int gy = min(max(y0 - R + hy, 0), ny - 1);
            const float* rowp = plane + (long long)gy * nx;
            const float v0 = __ldg(rowp + gxa), v1 = __ldg(rowp + gxa + a.ps_in),
                        v2 = __ldg(rowp + gxa + 2 * a.ps_in);
            float* t = tile + hy * HXP + tx;
            t[0] = v0;
            t[TILE] = v1;
            t[2 * TILE] = v2;
            if (second) {
                const float w0 = __ldg(rowp + gxb), w1 = __ldg(rowp + gxb + a.ps_in),
                            w2 = __ldg(rowp + gxb + 2 * a.ps_in);
                t[32] = w0;
                t[TILE + 32] = w1;
                t[2 * TILE + 32] = w2;
            }
        }
    }
    __syncthreads();
    // x pass: (component, halo row, group of four output columns)
    for (int s = tid; s < 3 * HY * (XY_T / 4); s += XY_NT) {
        const int c = s / (HY * (XY_T / 4)), rr = s - c * (HY * (XY_T / 4));
        const int hy = rr >> 3, g4 = rr & 7;
        const float4* row = reinterpret_cast<const float4*>(tile + c * TILE + hy * HXP) + g4;
        float win[4 * NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const float4 q = row[v];
            win[4 * v] = q.x;
            win[4 * v + 1] = q.y;
            win[4 * v + 2] = q.z;
            win[4 * v + 3] = q.w;
        }
        float4 o = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
        for (int t = 0; t <= 2 * R; ++t) {
            const float w = a.tx_[t];
            o.x = fmaf(w, win[t], o.x);
            o.y = fmaf(w, win[t + 1], o.y);
            o.z = fmaf(w, win[t + 2], o.z);
            o.w = fmaf(w, win[t + 3], o.w);
        }
        reinterpret_cast<float4*>(xs + (c * HY + hy) * XY_T)[g4] = o;
    }
    __syncthreads();
    // y pass: four consecutive output rows of the thread's column, per component
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float col[4 + 2 * R];
#pragma unroll
        for (int t = 0; t < 4 + 2 * R; ++t) col[t] = xs[(c * HY + ty * 4 + t) * XY_T + tx];
        float* dst = tmp + c * ps_tmp + zoff;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float acc = 0.0f;
#pragma unroll
            for (int t = 0; t <= 2 * R; ++t) acc = fmaf(a.ty_[t], col[q + t], acc);
            const int y = y0 + ty * 4 + q;
            if (x < nx && y < ny) dst[(long long)y * nx + x] = acc;
        }
    }
}

template <int R>
__global__ void __launch_bounds__(XY_NT) k_smooth_xy(SmoothArgs a, const float* __restrict__ in,
                                                     float* __restrict__ tmp, long long ps_tmp) {
    pdl_wait();
    extern __shared__ __align__(16) float smem_xy[];
    smooth_xy_tile<R>(a, blockIdx.x, blockIdx.y, blockIdx.z, smem_xy, in, tmp, ps_tmp);
}

// The xy pass of every active subject of a batch: input at in + b * stride (or at the subject's
// multichannel accumulator), output into tmp + b * stride; tiles (x, y, slice) in the single
// kernel's block order.
template <int R>
__global__ void __launch_bounds__(XY_NT) k_smooth_xy_batch(SmoothArgs a, BatchList L,
                                                           const float* __restrict__ in,
                                                           float* __restrict__ tmp,
                                                           long long stride) {
    extern __shared__ __align__(16) float smem_xy[];
    const int work = *L.count * L.tiles;
    const int gx = (a.g.nx + XY_T - 1) / XY_T, gy = (a.g.ny + XY_T - 1) / XY_T;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles];
        int bx, by, bz;
        tile_coords(w % L.tiles, gx, gy, bx, by, bz);
        smooth_xy_tile<R>(a, bx, by, bz, smem_xy, in + b * stride, tmp + b * stride, a.ps_out);
        __syncthreads();  // the next tile reloads the shared tile
    }
}

// The thread's column of tile (z segment zb, 32 columns xb, 8 rows yb) of the z pass; returns the
// largest |u/sp| it wrote (when max_bits is wanted).
template <int R>
__device__ __forceinline__ float smooth_z_tile(const SmoothArgs& a, int zb, int xb, int yb,
                                               const float* __restrict__ tmp, long long ps_tmp,
                                               const float* in, float* out, bool want_max) {
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int x = xb * 32 + (threadIdx.x & 31), y = yb * 8 + (threadIdx.x >> 5);
    const int zs = zb * Z_SEG;
    const long long sxy = (long long)nx * ny;
    float vmax = 0.0f;
    if (x < nx && y < ny) {
        const long long col = (long long)y * nx + x;
        const float isp[3] = {(float)(1.0 / a.g.sp[0]), (float)(1.0 / a.g.sp[1]),
                              (float)(1.0 / a.g.sp[2])};
        const bool edge_xy = x == 0 || y == 0 || x == nx - 1 || y == ny - 1;
        float nsq[Z_SEG];
#pragma unroll
        for (int q = 0; q < Z_SEG; ++q) nsq[q] = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float* src = tmp + c * ps_tmp + col;
            float w[Z_SEG + 2 * R];
#pragma unroll
            for (int t = 0; t < Z_SEG + 2 * R; ++t) {
                const int zz = min(max(zs - R + t, 0), nz - 1);  // edge replication
                w[t] = __ldg(src + zz * sxy);
            }
#pragma unroll
            for (int q = 0; q < Z_SEG; ++q) {
                const int z = zs + q;
                if (z >= nz) break;
                float v = 0.0f;
#pragma unroll
                for (int t = 0; t <= 2 * R; ++t) v = fmaf(a.tz_[t], w[q + t], v);
                const long long l = (long long)z * sxy + col;
                const bool face = edge_xy || z == 0 || z == nz - 1;
                float o;
                if (face) o = 0.0f;
                else if (a.w2 != 0.0f) o = v * a.w1 + in[l + c * a.ps_in] * a.w2;
                else o = v;
                out[l + c * a.ps_out] = o;
                const float p = o * isp[c];
                nsq[q] = fmaf(p, p, nsq[q]);
            }
        }
        if (want_max) {
#pragma unroll
            for (int q = 0; q < Z_SEG; ++q)
                if (zs + q < nz)
                    vmax = __int_as_float(max(__float_as_int(vmax),
                                              __float_as_int(nan_canon(sqrtf(nsq[q])))));
        }
    }
    return vmax;
}

// blockIdx.x: z segment (fastest, so neighbouring segments share their halo rows in L2),
// blockIdx.y: 32 columns in x, blockIdx.z: 8 rows in y.
template <int R>
__global__ void __launch_bounds__(256, R <= 6 ? 3 : 2) k_smooth_z(SmoothArgs a, const float* __restrict__ tmp,
                                                  long long ps_tmp, const float* in,
                                                  float* out,
                                                  unsigned int* __restrict__ max_bits) {
    pdl_wait();
    float vmax = smooth_z_tile<R>(a, blockIdx.x, blockIdx.y, blockIdx.z, tmp, ps_tmp, in, out,
                                  max_bits != nullptr);
    if (max_bits) {
        vmax = warp_max_f(vmax);
        if ((threadIdx.x & 31) == 0 && vmax > 0.0f) atomicMax(max_bits, __float_as_uint(vmax));
    }
}

// The z pass of every active subject of a batch: tmp / in / out at + b * stride, the max of
// subject b into max_bits[b * max_stride].
template <int R>
__global__ void __launch_bounds__(256) k_smooth_z_batch(SmoothArgs a, BatchList L,
                                                        const float* __restrict__ tmp,
                                                        const float* in, float* out,
                                                        long long stride,
                                                        unsigned int* __restrict__ max_bits,
                                                        int max_stride) {
    const int work = *L.count * L.tiles;
    const int gz = (a.g.nz + Z_SEG - 1) / Z_SEG, gx = (a.g.nx + 31) / 32;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles];
        int zb, xb, yb;
        tile_coords(w % L.tiles, gz, gx, zb, xb, yb);
        float vmax = smooth_z_tile<R>(a, zb, xb, yb, tmp + b * stride, a.ps_out, in + b * stride,
                                      out + b * stride, true);
        vmax = warp_max_f(vmax);
        if ((threadIdx.x & 31) == 0 && vmax > 0.0f)
            atomicMax(max_bits + b * max_stride, __float_as_uint(vmax));
    }
}

template <int R>
int launch_smooth_xyz(fw_ctx* ctx, const SmoothArgs& a, const fw_field* in, fw_field* out,
                      fw_field* tmp, unsigned int* d_max_bits) {
    constexpr int HY = XY_T + 2 * R, HXP = (XY_T + 2 * R + 3) & ~3, NV = (4 + 2 * R + 3) / 4;
    constexpr size_t bytes = sizeof(float) * (3 * HY * HXP + 4 * NV + 3 * HY * XY_T);
    FW_CUDA(cudaFuncSetAttribute(k_smooth_xy<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)bytes));
    dim3 g1((a.g.nx + XY_T - 1) / XY_T, (a.g.ny + XY_T - 1) / XY_T, a.g.nz);
    FW_TRY(launch_pdl(ctx, "k_smooth_xy", k_smooth_xy<R>, g1, dim3(XY_NT), bytes, a,
                      (const float*)in->d, tmp->d, (long long)tmp->ps));
    dim3 g2((a.g.nz + Z_SEG - 1) / Z_SEG, (a.g.nx + 31) / 32, (a.g.ny + 7) / 8);
    return launch_pdl(ctx, "k_smooth_z", k_smooth_z<R>, g2, dim3(256), 0, a,
                      (const float*)tmp->d, (long long)tmp->ps, (const float*)in->d, out->d,
                      d_max_bits);
}

template <int R>
int launch_smooth_batch_r(fw_ctx* ctx, const SmoothArgs& a, const int* active, const int* count,
                          int blocks_xy, int blocks_z, const float* in, float* out, float* tmp,
                          long long stride, unsigned int* max_bits, int max_stride) {
    constexpr int HY = XY_T + 2 * R, HXP = (XY_T + 2 * R + 3) & ~3, NV = (4 + 2 * R + 3) / 4;
    constexpr size_t bytes = sizeof(float) * (3 * HY * HXP + 4 * NV + 3 * HY * XY_T);
    FW_CUDA(cudaFuncSetAttribute(k_smooth_xy_batch<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)bytes));
    const int gx = (a.g.nx + XY_T - 1) / XY_T, gy = (a.g.ny + XY_T - 1) / XY_T;
    BatchList Lxy{active, count, gx * gy * a.g.nz};
    k_smooth_xy_batch<R><<<blocks_xy, XY_NT, bytes, ctx->stream>>>(a, Lxy, in, tmp, stride);
    FW_TRY(check_launch(ctx, "k_smooth_xy_batch"));
    const int gz = (a.g.nz + Z_SEG - 1) / Z_SEG, gxc = (a.g.nx + 31) / 32, gyc = (a.g.ny + 7) / 8;
    BatchList Lz{active, count, gz * gxc * gyc};
    k_smooth_z_batch<R><<<blocks_z, 256, 0, ctx->stream>>>(a, Lz, tmp, in, out, stride, max_bits,
                                                          max_stride);
    return check_launch(ctx, "k_smooth_z_batch");
}

// ---- Deriche recursive Gaussian (pyramid.rs:186-300, 418-427) --------------------------------

struct Deriche {
    double n[4], d[4], m[4], bn[4], bm[4];
};

int deriche_zero_order(double sigma, double spacing, Deriche& out) {
    if (spacing < 1e-8) return fail(FW_ERR_INVALID, "smoothing: spacing is too small");
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
    double smv = m1 + m2 + m3 + m4;
    sd = 1.0 + d1 + d2 + d3 + d4;
    double nn[4] = {n0, n1, n2, n3}, dd[4] = {d1, d2, d3, d4}, mm[4] = {m1, m2, m3, m4};
    for (int k = 0; k < 4; ++k) {
        out.n[k] = nn[k];
        out.d[k] = dd[k];
        out.m[k] = mm[k];
        out.bn[k] = dd[k] * sn / sd;
        out.bm[k] = dd[k] * smv / sd;
    }
    return 0;
}

// One thread per line along `axis` (pyramid.rs:240-300): the causal pass goes to `tmp`, the
// anticausal pass walks back with its last four inputs and outputs in registers and writes
// causal + anticausal to `out`. Lines of the y and z axes are coalesced across threads.
__global__ void k_deriche(const double* __restrict__ in, double* __restrict__ tmp,
                          double* __restrict__ out, int nx, int ny, int nz, int axis, Deriche c) {
    long long line = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long base, stride;
    int ln;
    if (axis == 0) {
        if (line >= (long long)ny * nz) return;
        base = line * nx;
        stride = 1;
        ln = nx;
    } else if (axis == 1) {
        if (line >= (long long)nx * nz) return;
        long long xq = line % nx, zq = line / nx;
        base = xq + zq * (long long)nx * ny;
        stride = nx;
        ln = ny;
    } else {
        if (line >= (long long)nx * ny) return;
        base = line;
        stride = (long long)nx * ny;
        ln = nz;
    }
    const double *n = c.n, *d = c.d, *m = c.m, *bn = c.bn, *bm = c.bm;
    const double* x = in + base;
    double* ca = tmp + base;
    double* o = out + base;
#define X(i) x[(long long)(i) * stride]
    double v1 = X(0);
    double c0 = X(0) * n[0] + v1 * n[1] + v1 * n[2] + v1 * n[3];
    double c1 = X(1) * n[0] + v1 * n[1] + v1 * n[2] + v1 * n[3];
    double c2 = X(2) * n[0] + X(1) * n[1] + v1 * n[2] + v1 * n[3];
    double c3 = X(3) * n[0] + X(2) * n[1] + X(1) * n[2] + v1 * n[3];
    c0 -= v1 * bn[0] + v1 * bn[1] + v1 * bn[2] + v1 * bn[3];
    c1 -= c0 * d[0] + v1 * bn[1] + v1 * bn[2] + v1 * bn[3];
    c2 -= c1 * d[0] + c0 * d[1] + v1 * bn[2] + v1 * bn[3];
    c3 -= c2 * d[0] + c1 * d[1] + c0 * d[2] + v1 * bn[3];
    ca[0] = c0;
    ca[stride] = c1;
    ca[2 * stride] = c2;
    ca[3 * stride] = c3;
    {
        double xm1 = X(3), xm2 = X(2), xm3 = X(1);
        double cm1 = c3, cm2 = c2, cm3 = c1, cm4 = c0;
        for (int i = 4; i < ln; ++i) {
            double xi = X(i);
            double ci = xi * n[0] + xm1 * n[1] + xm2 * n[2] + xm3 * n[3];
            ci -= cm1 * d[0] + cm2 * d[1] + cm3 * d[2] + cm4 * d[3];
            ca[(long long)i * stride] = ci;
            xm3 = xm2;
            xm2 = xm1;
            xm1 = xi;
            cm4 = cm3;
            cm3 = cm2;
            cm2 = cm1;
            cm1 = ci;
        }
    }
    double v2 = X(ln - 1);
    double e1 = v2 * m[0] + v2 * m[1] + v2 * m[2] + v2 * m[3];                   // an[ln-1]
    double e2 = X(ln - 1) * m[0] + v2 * m[1] + v2 * m[2] + v2 * m[3];            // an[ln-2]
    double e3 = X(ln - 2) * m[0] + X(ln - 1) * m[1] + v2 * m[2] + v2 * m[3];     // an[ln-3]
    double e4 = X(ln - 3) * m[0] + X(ln - 2) * m[1] + X(ln - 1) * m[2] + v2 * m[3];  // an[ln-4]
    e1 -= v2 * bm[0] + v2 * bm[1] + v2 * bm[2] + v2 * bm[3];
    e2 -= e1 * d[0] + v2 * bm[1] + v2 * bm[2] + v2 * bm[3];
    e3 -= e2 * d[0] + e1 * d[1] + v2 * bm[2] + v2 * bm[3];
    e4 -= e3 * d[0] + e2 * d[1] + e1 * d[2] + v2 * bm[3];
    o[(long long)(ln - 1) * stride] = ca[(long long)(ln - 1) * stride] + e1;
    o[(long long)(ln - 2) * stride] = ca[(long long)(ln - 2) * stride] + e2;
    o[(long long)(ln - 3) * stride] = ca[(long long)(ln - 3) * stride] + e3;
    o[(long long)(ln - 4) * stride] = ca[(long long)(ln - 4) * stride] + e4;
    // an[i-1] = x[i] m0 + x[i+1] m1 + x[i+2] m2 + x[i+3] m3 - (an[i] d0 + an[i+1] d1 + an[i+2] d2 + an[i+3] d3)
    double xp1 = X(ln - 3), xp2 = X(ln - 2), xp3 = X(ln - 1);  // x[i+1..i+3] at i = ln - 4
    double a0 = e4, a1 = e3, a2 = e2, a3 = e1;                 // an[i..i+3] at i = ln - 4
    for (int i = ln - 4; i >= 1; --i) {
        double xi = X(i);
        double an = xi * m[0] + xp1 * m[1] + xp2 * m[2] + xp3 * m[3];
        an -= a0 * d[0] + a1 * d[1] + a2 * d[2] + a3 * d[3];
        o[(long long)(i - 1) * stride] = ca[(long long)(i - 1) * stride] + an;
        xp3 = xp2;
        xp2 = xp1;
        xp1 = xi;
        a3 = a2;
        a2 = a1;
        a1 = a0;
        a0 = an;
    }
#undef X
}

__global__ void k_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, long long n) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l < n) b[l] = a[l];
}

__global__ void k_f64_to_f32(const double* __restrict__ a, float* __restrict__ b, long long n) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l < n) b[l] = (float)a[l];
}

}  // namespace

int launch_smooth(fw_ctx* ctx, const fw_field* in, fw_field* out, double variance,
                  unsigned int* d_max_bits, fw_field* tmp) {
    SmoothArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = dev_grid(in->grid);
    a.ps_in = in->ps;
    a.ps_out = out->ps;
    int r[3];
    for (int ax = 0; ax < 3; ++ax) {
        std::vector<double> k = gaussian_taps(variance, 0.001, in->grid.n[ax]);
        int rad = (int)k.size() / 2;
        if (rad > (MAX_TAPS - 1) / 2)
            return fail(FW_ERR_INVALID, "smooth field: the Gaussian kernel radius exceeds 24 voxels");
        r[ax] = rad;
        float* dst = ax == 0 ? a.tx_ : (ax == 1 ? a.ty_ : a.tz_);
        for (size_t t = 0; t < k.size(); ++t) dst[t] = (float)k[t];
    }
    a.rx = r[0];
    a.ry = r[1];
    a.rz = r[2];
    double w1 = variance < 0.5 ? 1.0 - variance / 0.5 : 1.0;
    a.w1 = (float)w1;
    a.w2 = (float)(1.0 - w1);
    bool same = tmp != nullptr && r[0] == r[1] && r[1] == r[2];
    for (int t = 0; same && t <= 2 * r[0]; ++t)
        same = a.tx_[t] == a.ty_[t] && a.ty_[t] == a.tz_[t];
    if (same) {
        FW_CHECK(tmp->grid.same(in->grid) && tmp != in && tmp != out,
                 "smooth field: the temporary field must be a third field on the same grid");
        switch (r[0]) {
            case 1: return launch_smooth_xyz<1>(ctx, a, in, out, tmp, d_max_bits);
            case 2: return launch_smooth_xyz<2>(ctx, a, in, out, tmp, d_max_bits);
            case 3: return launch_smooth_xyz<3>(ctx, a, in, out, tmp, d_max_bits);
            case 4: return launch_smooth_xyz<4>(ctx, a, in, out, tmp, d_max_bits);
            case 5: return launch_smooth_xyz<5>(ctx, a, in, out, tmp, d_max_bits);
            case 6: return launch_smooth_xyz<6>(ctx, a, in, out, tmp, d_max_bits);
            case 7: return launch_smooth_xyz<7>(ctx, a, in, out, tmp, d_max_bits);
            case 8: return launch_smooth_xyz<8>(ctx, a, in, out, tmp, d_max_bits);
            case 9: return launch_smooth_xyz<9>(ctx, a, in, out, tmp, d_max_bits);
            case 10: return launch_smooth_xyz<10>(ctx, a, in, out, tmp, d_max_bits);
            case 11: return launch_smooth_xyz<11>(ctx, a, in, out, tmp, d_max_bits);
            case 12: return launch_smooth_xyz<12>(ctx, a, in, out, tmp, d_max_bits);
            default: break;
        }
    }
    FW_CHECK(in != out, "smooth field: the general path needs a separate output");
    dim3 grid((a.g.nx + STX - 1) / STX, (a.g.ny + STY - 1) / STY, 1);
    long long tiles = (long long)grid.x * grid.y;
    int want = (int)std::max<long long>(1, (4LL * ctx->num_sms + tiles - 1) / tiles);
    int chunk = (a.g.nz + want - 1) / want;
    chunk = std::max(chunk, std::min(a.g.nz, 4 * a.rz + 4));
    a.zchunk = chunk;
    grid.z = (a.g.nz + chunk - 1) / chunk;
    const int HX = STX + 2 * a.rx, HY = STY + 2 * a.ry, W = 2 * a.rz + 1;
    size_t bytes = sizeof(float) * (3 * HY * HX + 3 * HY * STX + W * 3 * SNT);
    FW_CUDA(cudaFuncSetAttribute(k_smooth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    k_smooth<<<grid, SNT, bytes, ctx->stream>>>(a, in->d, out->d, d_max_bits);
    return check_launch(ctx, "k_smooth");
}

int launch_smooth_batch(fw_ctx* ctx, const HostGrid& g, long long ps, double variance,
                        const int* active, const int* count, int blocks_xy, int blocks_z,
                        const float* in, float* out, float* tmp, long long stride,
                        unsigned int* max_bits, int max_stride) {
    SmoothArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = dev_grid(g);
    a.ps_in = a.ps_out = ps;
    int r[3];
    for (int ax = 0; ax < 3; ++ax) {
        std::vector<double> k = gaussian_taps(variance, 0.001, g.n[ax]);
        r[ax] = (int)k.size() / 2;
        if (r[ax] > 12)
            return fail(FW_ERR_INVALID, "batched SyN: the update field's Gaussian radius exceeds 12");
        float* dst = ax == 0 ? a.tx_ : (ax == 1 ? a.ty_ : a.tz_);
        for (size_t t = 0; t < k.size(); ++t) dst[t] = (float)k[t];
    }
    bool same = r[0] == r[1] && r[1] == r[2];
    for (int t = 0; same && t <= 2 * r[0]; ++t)
        same = a.tx_[t] == a.ty_[t] && a.ty_[t] == a.tz_[t];
    if (!same)
        return fail(FW_ERR_INVALID,
                    "batched SyN: the update field's Gaussian differs between axes on this grid");
    a.rx = a.ry = a.rz = r[0];
    double w1 = variance < 0.5 ? 1.0 - variance / 0.5 : 1.0;
    a.w1 = (float)w1;
    a.w2 = (float)(1.0 - w1);
#define FW_SMOOTH_BATCH(RR) \
    case RR:                \
        return launch_smooth_batch_r<RR>(ctx, a, active, count, blocks_xy, blocks_z, in, out, tmp, stride, max_bits, max_stride);
    switch (r[0]) {
        FW_SMOOTH_BATCH(1)
        FW_SMOOTH_BATCH(2)
        FW_SMOOTH_BATCH(3)
        FW_SMOOTH_BATCH(4)
        FW_SMOOTH_BATCH(5)
        FW_SMOOTH_BATCH(6)
        FW_SMOOTH_BATCH(7)
        FW_SMOOTH_BATCH(8)
        FW_SMOOTH_BATCH(9)
        FW_SMOOTH_BATCH(10)
        FW_SMOOTH_BATCH(11)
        FW_SMOOTH_BATCH(12)
        default:
            return fail(FW_ERR_INVALID, "batched SyN: the update field's Gaussian radius is zero");
    }
#undef FW_SMOOTH_BATCH
}

int launch_smooth_recursive(fw_ctx* ctx, const fw_image* img, const double sigma_mm[3],
                            fw_image* out) {
    const HostGrid& g = img->grid;
    long long n = g.count();
    for (int ax = 0; ax < 3; ++ax) {
        if (g.n[ax] < 4) return fail(FW_ERR_INVALID, "smoothing: an axis has fewer than 4 voxels");
        if (!(sigma_mm[ax] > 0.0)) return fail(FW_ERR_INVALID, "smoothing: sigma must be greater than zero");
    }
    double *vol = nullptr, *tmp = nullptr, *nxt = nullptr;
    FW_TRY(dev_alloc(ctx, sizeof(double) * n, (void**)&vol));
    int rc = dev_alloc(ctx, sizeof(double) * n, (void**)&tmp);
    if (!rc) rc = dev_alloc(ctx, sizeof(double) * n, (void**)&nxt);
    if (rc) {
        dev_free(ctx, vol, sizeof(double) * n);
        dev_free(ctx, tmp, sizeof(double) * n);
        return rc;
    }
    unsigned int blocks = (unsigned int)((n + 255) / 256);
    k_f32_to_f64<<<blocks, 256, 0, ctx->stream>>>(img->d, vol, n);
    rc = check_launch(ctx, "k_f32_to_f64");
    const int order[3] = {2, 0, 1};  // SmoothingRecursiveGaussianImageFilter: z, x, y
    for (int oi = 0; oi < 3 && !rc; ++oi) {
        int ax = order[oi];
        Deriche c;
        rc = deriche_zero_order(sigma_mm[ax], g.sp[ax], c);
        if (rc) break;
        long long lines = n / g.n[ax];
        k_deriche<<<(unsigned int)((lines + 127) / 128), 128, 0, ctx->stream>>>(
            vol, tmp, nxt, (int)g.n[0], (int)g.n[1], (int)g.n[2], ax, c);
        rc = check_launch(ctx, "k_deriche");
        std::swap(vol, nxt);
    }
    if (!rc) {
        k_f64_to_f32<<<blocks, 256, 0, ctx->stream>>>(vol, out->d, n);
        rc = check_launch(ctx, "k_f64_to_f32");
    }
    dev_free(ctx, vol, sizeof(double) * n);
    dev_free(ctx, tmp, sizeof(double) * n);
    dev_free(ctx, nxt, sizeof(double) * n);
    return rc;
}

}  // namespace fw

using namespace fw;

extern "C" {

int fw_smooth_field(fw_ctx* ctx, fw_field* field, double variance) {
    FW_CHECK(ctx && field, "null argument");
    if (!(variance > 0.0)) return 0;  // returned unchanged (faces not zeroed)
    fw_field *tmp = nullptr, *res = nullptr;
    FW_TRY(new_field(ctx, field->grid, &tmp));
    int rc = new_field(ctx, field->grid, &res);
    // the result lands in `res` (tmp holds the xy pass), then takes the field's place
    if (!rc) rc = launch_smooth(ctx, field, res, variance, nullptr, tmp);
    if (!rc) {
        std::swap(field->d, res->d);
        rc = sync(ctx);
    }
    fw_field_free(res);
    fw_field_free(tmp);
    return rc;
}

int fw_smooth_recursive(fw_ctx* ctx, const fw_image* img, const double sigma_mm[3],
                        fw_image** out) {
    FW_CHECK(ctx && img && sigma_mm && out, "null argument");
    fw_image* im;
    FW_TRY(new_image(ctx, img->grid, &im));
    int rc = launch_smooth_recursive(ctx, img, sigma_mm, im);
    if (!rc) rc = sync(ctx);
    if (rc) {
        fw_image_free(im);
        return rc;
    }
    *out = im;
    return 0;
}

}  // extern "C"
