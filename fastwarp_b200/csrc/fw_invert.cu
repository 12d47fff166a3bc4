// fw_invert.cu -- ITK InvertDisplacementFieldImageFilter as SyN runs it (field_ops.rs:309-392).
//
// The reference loop is: while (iteration < max && max_error > max_tol && mean_error > mean_tol)
// { e = psi + f(x + psi); measure mean and max of |e/sp|; psi += eps * clamp(-e) with
// eps = 0.75 on the first body and 0.5 after; faces of psi to zero }.
//
// Device design: the error at voxel x depends only on psi(x) and the read-only field f, so the
// sweep that measures a body's error can apply the same body's update to psi(x) in place -- the
// only thing it cannot know yet is the clamp, which needs the body's maximum error over the whole
// volume. A body is therefore three kernels:
//   k_inv_bound  the error on a sparse lattice of voxels (one in 64): its maximum is a lower
//                bound L on the body's maximum error;
//   k_inv_step   the measurement over 32 x 8 x 2 column tiles, each thread keeping its column's
//                psi and error in registers. No voxel of a warp's part (32 columns of a row,
//                2 slices) whose largest error is at most eps * L can be clamped (eps * L <=
//                eps * max), so such a part updates psi in place at once; any other part writes
//                its errors to the residual field and enters a short list. A fixed-order
//                reduction (the last block) gives the mean and max and decides whether another
//                body runs;
//   k_inv_fix    the listed parts' updates, now with the clamp eps * max.
// The update of every voxel is the same arithmetic on either path, so the result does not depend
// on which parts were deferred. The loop state lives in device memory, so the loop needs no host
// read-back: the SyN driver runs it inside a CUDA graph WHILE node whose condition the step's last
// block sets. The batched kernels (many subjects, one launch each) run the same three kernels'
// bodies over a work list of (subject, block) items.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>

#include "fw_internal.cuh"

namespace fw {

struct InvArgs {
    DevGrid g;
    long long ps_f, ps_psi;
    float isx, isy, isz;
    int zchunk;  // step tiles stacked in a block (k_inv_step)
};

// e = psi + f(x + psi) at voxel (i, j, k) with psi = (px, py, pz) (field_ops.rs:346-351).
__device__ __forceinline__ void residual(const InvArgs& a, const float* __restrict__ f, int i,
                                         int j, int k, float px, float py, float pz, float e[3]) {
    // explicitly rounded (no contraction), in the reference's order: every kernel that measures
    // a voxel maps it to the same continuous index
    auto map = [&](int r, int base) {
        const double* m = a.g.inv + 3 * r;
        return __dadd_rn((double)base, __dadd_rn(__dadd_rn(__dmul_rn(m[0], (double)px),
                                                           __dmul_rn(m[1], (double)py)),
                                                 __dmul_rn(m[2], (double)pz)));
    };
    const double c0 = map(0, i), c1 = map(1, j), c2 = map(2, k);
    float d[3] = {0.0f, 0.0f, 0.0f};
    if (inside_index(c0, c1, c2, a.g.nx, a.g.ny, a.g.nz))
        vec_at_index(f, a.ps_f, a.g.nx, a.g.ny, a.g.nz, c0, c1, c2, d);
    e[0] = px + d[0];
    e[1] = py + d[1];
    e[2] = pz + d[2];
}

// |e / sp| of one voxel's error (every kernel that measures a voxel uses this one expression).
// In a SyN run's first iteration the largest error equals the gradient step up to rounding, so
// with a step of 0.1 (the inversion's max-error tolerance) this float's last bit decides whether
// a second body runs; the expression is the one validated against the oracle.
__device__ __forceinline__ float err_norm(const InvArgs& a, const float e[3]) {
    const float x = e[0] * a.isx, y = e[1] * a.isy, z = e[2] * a.isz;
    return sqrtf(x * x + y * y + z * z);
}

// psi + eps * clamp(-e) at one voxel (field_ops.rs:368-383), faces to zero with `enforce`.
__device__ __forceinline__ void update_voxel(const InvArgs& a, int i, int j, int k, float nrm,
                                             const float e[3], float eps, float limit,
                                             bool enforce, float p[3]) {
    float ux = -e[0], uy = -e[1], uz = -e[2];
    if (nrm > limit) {
        const float fct = limit / nrm;
        ux *= fct;
        uy *= fct;
        uz *= fct;
    }
    p[0] = p[0] + ux * eps;
    p[1] = p[1] + uy * eps;
    p[2] = p[2] + uz * eps;
    const bool face = i == 0 || j == 0 || k == 0 || i == a.g.nx - 1 || j == a.g.ny - 1 ||
                      k == a.g.nz - 1;
    if (enforce && face) p[0] = p[1] = p[2] = 0.0f;
}

// Block sums (f64) and maxima -> partials; the last block reduces them in block order and
// updates the loop state through `finish`.
// `bid` of `nblocks`: the tile (or virtual block) whose partials these are.
template <typename Finish>
__device__ void reduce_and_finish(double sum, float mx, double* __restrict__ partials,
                                  unsigned int* __restrict__ counter, unsigned int bid,
                                  unsigned int nblocks, Finish finish) {
    __shared__ double rs[32];
    __shared__ float rm[32];
    __shared__ bool last;
    sum = warp_sum_d(sum);
    mx = warp_max_f(mx);
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        rs[w] = sum;
        rm[w] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        float m = 0.0f;
        for (int q = 0; q < nw; ++q) {
            s += rs[q];
            m = __int_as_float(max(__float_as_int(m), __float_as_int(rm[q])));
        }
        partials[2 * bid] = s;
        partials[2 * bid + 1] = (double)m;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == nblocks - 1;
    __syncthreads();
    if (!last) return;
    // the whole last block reduces the partials in a fixed order
    __shared__ double red[32];
    const double s = block_sum_fixed(partials, nblocks, 2, red);
    const double m = block_max_nan(partials + 1, nblocks, 2, red);
    if (threadIdx.x == 0) {
        finish(s, m);
        *counter = 0;
    }
}

// ---- one inversion body: bound, step, fix --------------------------------------------------

#ifndef FW_STEP_Z
#define FW_STEP_Z 2
#endif
#ifndef FW_STEP_MIN_BLOCKS
#define FW_STEP_MIN_BLOCKS 4
#endif
#ifndef FW_STEP_MAX_TILES
#define FW_STEP_MAX_TILES 8
#endif
#ifndef FW_BOUND_STRIDE
#define FW_BOUND_STRIDE 4
#endif
constexpr int kStepZ = FW_STEP_Z;  // slices of a step tile (a thread's column stays in registers)
// eps * L is lowered by this factor before tiles are compared with it: the bound and the step
// measure a voxel with the same code, so L is one of the step's errors; the factor guards against
// the compiler contracting the norm's products differently in the two kernels (a last-bit change)
constexpr float kSafeMargin = 0.999f;

// The loop's settings before its first body (field_ops.rs:330-344: errors start at +inf, so the
// first body runs whenever max_iterations > 0).
__device__ __forceinline__ void init_state(InvState* __restrict__ st, const fw_invert_params& prm) {
    st->max_iterations = prm.max_iterations;
    st->mean_tol = prm.mean_error_tolerance;
    st->max_tol = prm.max_error_tolerance;
    st->enforce = prm.enforce_boundary_condition;
    st->mean = 0.0;
    st->max = 0.0;
    st->executed = 0;
    st->k = 0;
    st->go = prm.max_iterations > 0 ? 1 : 0;
    st->lb = 0u;
    st->ndefer = 0u;
    st->eps = 0.0f;
    st->limit = 0.0f;
}

__global__ void k_inv_init(InvState* __restrict__ st, fw_invert_params prm,
                           cudaGraphConditionalHandle handle, int use_handle) {
    init_state(st, prm);
    if (use_handle) cudaGraphSetConditional(handle, st->go ? 1u : 0u);
}

// Several inversions' settings in one launch: states st[0..count) and the conditions of their
// WHILE nodes; it also clears zero[0..nzero) (the SyN level graph begins every iteration with it:
// its four inversions' settings and the update maxima, in one node).
struct InitHandles {
    cudaGraphConditionalHandle h[kMaxInitHandles];
};
__global__ void k_inv_init_many(InvState* __restrict__ st, int count, fw_invert_params prm,
                                InitHandles hs, unsigned int* __restrict__ zero, int nzero) {
    pdl_wait();
    const int i = threadIdx.x;
    if (i < count) {
        init_state(st + i, prm);
        cudaGraphSetConditional(hs.h[i], st[i].go ? 1u : 0u);
    }
    if (i < nzero) zero[i] = 0u;
}

// The lattice of the bound: voxels 1, 1 + S, 1 + 2S, ... along each axis (0 on an axis of one
// voxel), S = kBoundStride.
constexpr int kBoundStride = FW_BOUND_STRIDE;
struct Lattice {
    int ox, oy, oz, mx, my, mz;
    __host__ __device__ long long count() const { return (long long)mx * my * mz; }
};

static Lattice lattice_of(const DevGrid& g) {
    constexpr int S = kBoundStride;
    Lattice t;
    t.ox = g.nx > 1 ? 1 : 0;
    t.oy = g.ny > 1 ? 1 : 0;
    t.oz = g.nz > 1 ? 1 : 0;
    t.mx = (g.nx - t.ox + S - 1) / S;
    t.my = (g.ny - t.oy + S - 1) / S;
    t.mz = (g.nz - t.oz + S - 1) / S;
    return t;
}

// The running body's error on the lattice points vb, vb + nvb, ... (256 a block step) of one
// inverse; the block's largest (as float bits, NaN above everything) goes into st->lb, the lower
// bound L the step compares tiles with.
__device__ __forceinline__ void bound_block(const InvArgs& a, const Lattice& t,
                                            const float* __restrict__ f,
                                            const float* __restrict__ psi,
                                            InvState* __restrict__ st, unsigned int vb,
                                            unsigned int nvb) {
    __shared__ float wm[8];
    float best = 0.0f;
    const long long m = t.count();
    for (long long s = (long long)vb * blockDim.x + threadIdx.x; s < m;
         s += (long long)nvb * blockDim.x) {
        const long long q = s / t.mx;
        const int i = t.ox + kBoundStride * (int)(s - q * t.mx);
        const int j = t.oy + kBoundStride * (int)(q % t.my);
        const int k = t.oz + kBoundStride * (int)(q / t.my);
        const long long l = ((long long)k * a.g.ny + j) * a.g.nx + i;
        float e[3];
        residual(a, f, i, j, k, psi[l], psi[l + a.ps_psi], psi[l + 2 * a.ps_psi], e);
        const float nrm = nan_canon(err_norm(a, e));
        best = __int_as_float(max(__float_as_int(best), __float_as_int(nrm)));
    }
    best = warp_max_f(best);
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w)
            best = __int_as_float(max(__float_as_int(best), __float_as_int(wm[w])));
        atomicMax(&st->lb, __float_as_uint(best));
    }
    __syncthreads();  // wm is free for the block's next item
}

// The bound of the running body (also clears the previous body's deferred list, whose fix
// kernel has run).
__global__ void __launch_bounds__(256) k_inv_bound(InvArgs a, Lattice t, const float* __restrict__ f,
                                                   const float* __restrict__ psi,
                                                   InvState* __restrict__ st) {
    pdl_wait();
    if (blockIdx.x == 0 && threadIdx.x == 0) st->ndefer = 0u;
    if (!st->go) return;
    bound_block(a, t, f, psi, st, blockIdx.x, gridDim.x);
}

// A warp's part of step tile (bx, by, bz) -- 32 columns of one row, kStepZ slices: each thread's
// column is measured with psi and e in registers, and the warp's largest error decides whether it
// updates psi now (no voxel of it can exceed eps * L <= the clamp) or keeps its errors in `res`
// for the fix kernel. No block barrier: every warp decides alone. Returns whether the warp's
// voxels were deferred (uniform over the warp).
__device__ __forceinline__ bool step_warp(const InvArgs& a, int bx, int by, int bz,
                                          const float* __restrict__ f, float* __restrict__ psi,
                                          float* __restrict__ res, float eps, float safe,
                                          bool enforce, double& sum, float& mx) {
    int x, y, z0, z1;
    const bool have = column_of_tile(a.g.nx, a.g.ny, a.g.nz, kStepZ, bx, by, bz, x, y, z0, z1);
    const long long sxy = (long long)a.g.nx * a.g.ny;
    const long long l0 = (long long)z0 * sxy + (long long)y * a.g.nx + x;
    float p[kStepZ][3], e[kStepZ][3];
    float tmax = 0.0f;
    if (have) {
#pragma unroll
        for (int q = 0; q < kStepZ; ++q) {
            if (z0 + q < z1) {
                const long long l = l0 + q * sxy;
                p[q][0] = psi[l];
                p[q][1] = psi[l + a.ps_psi];
                p[q][2] = psi[l + 2 * a.ps_psi];
            }
        }
#pragma unroll
        for (int q = 0; q < kStepZ; ++q) {
            if (z0 + q < z1) {
                residual(a, f, x, y, z0 + q, p[q][0], p[q][1], p[q][2], e[q]);
                const float nrm = nan_canon(err_norm(a, e[q]));
                sum += (double)nrm;
                tmax = __int_as_float(max(__float_as_int(tmax), __float_as_int(nrm)));
            }
        }
    }
    mx = __int_as_float(max(__float_as_int(mx), __float_as_int(tmax)));
    const bool now = warp_max_f(tmax) <= safe;  // false when either is NaN
    if (have) {
#pragma unroll
        for (int q = 0; q < kStepZ; ++q) {
            if (z0 + q < z1) {
                const long long l = l0 + q * sxy;
                if (now) {
                    // the clamp cannot apply: limit = eps * max >= eps * L >= every error here
                    update_voxel(a, x, y, z0 + q, 0.0f, e[q], eps, 1.0f, enforce, p[q]);
                    psi[l] = p[q][0];
                    psi[l + a.ps_psi] = p[q][1];
                    psi[l + 2 * a.ps_psi] = p[q][2];
                } else {
                    res[l] = e[q][0];
                    res[l + a.ps_psi] = e[q][1];
                    res[l + 2 * a.ps_psi] = e[q][2];
                }
            }
        }
    }
    return !now;
}

// Block (bx, by, bzb) of body k's step: a.zchunk step tiles one above the other, measured against
// f (sum and max added to sum / mx), each warp's part updated at once or listed in `defer`
// (entries index the warp parts of the grid: gx columns of 32, every row y, ceil(nz / kStepZ)
// slices of kStepZ).
__device__ __forceinline__ void step_block(const InvArgs& a, int bx, int by, int bzb, int gx,
                                           const float* __restrict__ f,
                                           float* __restrict__ psi, float* __restrict__ res,
                                           InvState* __restrict__ st,
                                           unsigned int* __restrict__ defer, double& sum,
                                           float& mx) {
    const int kb = st->k;
    const float eps = kb == 0 ? 0.75f : 0.5f;
    const float safe = __fmul_rn(__fmul_rn(eps, __uint_as_float(st->lb)), kSafeMargin);
    const bool enforce = st->enforce != 0;
    const int gz = (a.g.nz + kStepZ - 1) / kStepZ;
    const int y = by * 8 + (threadIdx.x >> 5);
    const unsigned int cap = (unsigned int)gx * (unsigned int)a.g.ny * (unsigned int)gz;
    for (int m = 0; m < a.zchunk; ++m) {
        const int tz = bzb * a.zchunk + m;
        if (tz >= gz) break;  // uniform
        const bool deferred = step_warp(a, bx, by, tz, f, psi, res, eps, safe, enforce, sum, mx);
        if (deferred && (threadIdx.x & 31) == 0 && y < a.g.ny) {
            const unsigned int at = atomicAdd(&st->ndefer, 1u);
            if (at < cap)
                defer[at] = (unsigned int)bx +
                            (unsigned int)gx * ((unsigned int)y + (unsigned int)a.g.ny * tz);
        }
    }
}

// The last block's record of body k (field_ops.rs:339-355): errors, bodies executed, the step
// and clamp the fix kernel applies, and whether body k + 1 runs.
__device__ __forceinline__ bool finish_step(InvState* __restrict__ st, double s, double m,
                                            double count) {
    const int kb = st->k;
    const float eps = kb == 0 ? 0.75f : 0.5f;
    const double mean = s / count;
    const bool next = (kb + 1 < st->max_iterations) && m > st->max_tol && mean > st->mean_tol;
    st->mean = mean;
    st->max = m;
    st->executed = kb + 1;
    st->k = kb + 1;
    st->eps = eps;
    st->limit = eps * (float)m;
    st->lb = 0u;
    st->go = next ? 1 : 0;
    return next;
}

// Body k of the loop: measurement of psi against f (its mean and max), the update of every tile
// that cannot be clamped, and the list of the others. A block takes a.zchunk step tiles one above
// the other (fewer block partials on big grids); the last block reduces the partials in a fixed
// order, records the body and decides whether body k + 1 runs.
__global__ void __launch_bounds__(256, FW_STEP_MIN_BLOCKS) k_inv_step(InvArgs a, const float* __restrict__ f,
                                                     float* __restrict__ psi,
                                                     float* __restrict__ res,
                                                     double* __restrict__ partials,
                                                     unsigned int* __restrict__ counter,
                                                     InvState* __restrict__ st,
                                                     unsigned int* __restrict__ defer,
                                                     cudaGraphConditionalHandle handle,
                                                     int use_handle) {
    pdl_wait();
    if (!st->go) {  // uniform: the state only changes in the last block of a working grid
        if (use_handle && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 &&
            threadIdx.x == 0)
            cudaGraphSetConditional(handle, 0u);
        return;
    }
    double sum = 0.0;
    float mx = 0.0f;
    step_block(a, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, f, psi, res, st, defer, sum, mx);
    const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const unsigned int nblocks = gridDim.x * gridDim.y * gridDim.z;
    reduce_and_finish(sum, mx, partials, counter, bid, nblocks, [&](double s, double m) {
        const bool next = finish_step(st, s, m, (double)a.g.n);
        if (use_handle) cudaGraphSetConditional(handle, next ? 1u : 0u);
    });
}

// The deferred warp parts of the body that just ran, entries vb * 8 + w, + 8 nvb, ... of the list
// for warp w of the block: each voxel's update from its kept error, with the clamp at eps * max
// (field_ops.rs:368-383). Each voxel is written by one thread.
__device__ __forceinline__ void fix_tiles(const InvArgs& a, float* __restrict__ psi,
                                          const float* __restrict__ res,
                                          const InvState* __restrict__ st,
                                          const unsigned int* __restrict__ defer, unsigned int vb,
                                          unsigned int nvb) {
    const unsigned int gx = (unsigned int)(a.g.nx + 31) / 32, ny = (unsigned int)a.g.ny;
    const unsigned int cap = gx * ny * (unsigned int)((a.g.nz + kStepZ - 1) / kStepZ);
    const unsigned int n = min(st->ndefer, cap);
    if (n == 0u) return;
    const float eps = st->eps, limit = st->limit;
    const bool enforce = st->enforce != 0;
    const long long sxy = (long long)a.g.nx * a.g.ny;
    const unsigned int warps = blockDim.x >> 5;
    for (unsigned int t = vb * warps + (threadIdx.x >> 5); t < n; t += nvb * warps) {
        const unsigned int id = defer[t];
        const int x = (int)(id % gx) * 32 + (threadIdx.x & 31);
        const unsigned int r = id / gx;
        const int y = (int)(r % ny), z0 = (int)(r / ny) * kStepZ;
        if (x >= a.g.nx) continue;
        const int z1 = min(z0 + kStepZ, a.g.nz);
        for (int z = z0; z < z1; ++z) {
            const long long l = (long long)z * sxy + (long long)y * a.g.nx + x;
            const float e[3] = {res[l], res[l + a.ps_psi], res[l + 2 * a.ps_psi]};
            float p[3] = {psi[l], psi[l + a.ps_psi], psi[l + 2 * a.ps_psi]};
            update_voxel(a, x, y, z, err_norm(a, e), e, eps, limit, enforce, p);
            psi[l] = p[0];
            psi[l + a.ps_psi] = p[1];
            psi[l + 2 * a.ps_psi] = p[2];
        }
    }
}

__global__ void __launch_bounds__(256, 4) k_inv_fix(InvArgs a, float* __restrict__ psi,
                                                    const float* __restrict__ res,
                                                    const InvState* __restrict__ st,
                                                    const unsigned int* __restrict__ defer) {
    pdl_wait();
    fix_tiles(a, psi, res, st, defer, blockIdx.x, gridDim.x);
}

// ---- batched inversions: every active subject of a batch, each with its own loop state ------
//
// Subject b's field, inverse and residual are at f / psi / res + b * stride, its partials at
// partials + b * part_stride, its last-item counter at counter[b], its deferred list at
// defer + b * defer_stride and its loop state at st[b * st_stride]. A subject's items are the
// single kernels' blocks (the step's a.zchunk tiles each) and its partials are reduced in the
// same order, so its loop takes the same decisions as alone. The loop's condition is set
// afterwards by k_inv_any (any active subject still iterating).

__global__ void k_inv_init_batch(BatchList L, InvState* __restrict__ st, int st_stride,
                                 fw_invert_params prm) {
    const int n = *L.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        init_state(st + L.active[i] * st_stride, prm);
}

__global__ void __launch_bounds__(256) k_inv_bound_batch(InvArgs a, Lattice t, BatchList L,
                                                         const float* __restrict__ f,
                                                         const float* __restrict__ psi,
                                                         long long stride,
                                                         InvState* __restrict__ st,
                                                         int st_stride) {
    const int work = *L.count * L.tiles;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles];
        const unsigned int vb = (unsigned int)(w % L.tiles);
        InvState* sb = st + b * st_stride;
        if (vb == 0 && threadIdx.x == 0) sb->ndefer = 0u;
        if (!sb->go) continue;  // uniform
        bound_block(a, t, f + b * stride, psi + b * stride, sb, vb, (unsigned int)L.tiles);
    }
}

__global__ void __launch_bounds__(256, FW_STEP_MIN_BLOCKS) k_inv_step_batch(
    InvArgs a, BatchList L, const float* __restrict__ f, float* __restrict__ psi,
    float* __restrict__ res, long long stride, double* __restrict__ partials,
    long long part_stride, unsigned int* __restrict__ counter, InvState* __restrict__ st,
    int st_stride, unsigned int* __restrict__ defer, long long defer_stride) {
    const int work = *L.count * L.tiles;
    const int gx = (a.g.nx + 31) / 32, gy = (a.g.ny + 7) / 8;
    const double count = (double)a.g.n;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles], t = w % L.tiles;
        InvState* sb = st + b * st_stride;
        // uniform over the block; the state only changes once every item of the subject is done
        if (!sb->go) continue;
        int bx, by, bzb;
        tile_coords(t, gx, gy, bx, by, bzb);
        double sum = 0.0;
        float mx = 0.0f;
        step_block(a, bx, by, bzb, gx, f + b * stride, psi + b * stride, res + b * stride,
                   sb, defer + b * defer_stride, sum, mx);
        reduce_and_finish(sum, mx, partials + b * part_stride, counter + b, (unsigned int)t,
                          (unsigned int)L.tiles,
                          [&](double sm, double m) { finish_step(sb, sm, m, count); });
        __syncthreads();  // the next item reuses the reduction's shared memory
    }
}

__global__ void __launch_bounds__(256, 4) k_inv_fix_batch(InvArgs a, BatchList L,
                                                          float* __restrict__ psi,
                                                          const float* __restrict__ res,
                                                          long long stride,
                                                          const InvState* __restrict__ st,
                                                          int st_stride,
                                                          const unsigned int* __restrict__ defer,
                                                          long long defer_stride) {
    const int work = *L.count * L.tiles;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles];
        fix_tiles(a, psi + b * stride, res + b * stride, st + b * st_stride,
                  defer + b * defer_stride, (unsigned int)(w % L.tiles), (unsigned int)L.tiles);
    }
}

// The inner loop's condition: whether any active subject's inversion runs another body.
__global__ void k_inv_any(const InvState* __restrict__ st, int st_stride, BatchList L,
                          cudaGraphConditionalHandle handle) {
    const int n = *L.count;
    int any = 0;
    for (int i = threadIdx.x; i < n; i += 32) any |= st[L.active[i] * st_stride].go;
    any = __any_sync(0xffffffffu, any);
    if (threadIdx.x == 0) cudaGraphSetConditional(handle, any ? 1u : 0u);
}

static InvArgs inv_args(const fw_field* field, const fw_field* inverse) {
    InvArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = dev_grid(field->grid);
    a.ps_f = field->ps;
    a.ps_psi = inverse->ps;
    a.isx = (float)(1.0 / field->grid.sp[0]);
    a.isy = (float)(1.0 / field->grid.sp[1]);
    a.isz = (float)(1.0 / field->grid.sp[2]);
    return a;
}

// Step tiles per block on a grid: one unless the grid has more than about eight tiles an SM, then
// up to four (the last block's fixed-order reduction reads two doubles a block).
int inv_step_zchunk(const int64_t n[3], int num_sms) {
    const long long tiles = ((n[0] + 31) / 32) * ((n[1] + 7) / 8) * ((n[2] + kStepZ - 1) / kStepZ);
    return (int)std::max<long long>(1, std::min<long long>(FW_STEP_MAX_TILES, tiles / (8LL * num_sms)));
}

long long inv_step_parts(const HostGrid& g) {
    return (long long)((g.n[0] + 31) / 32) * g.n[1] * ((g.n[2] + kStepZ - 1) / kStepZ);
}

long long inv_step_tiles(const HostGrid& g) {
    return (long long)((g.n[0] + 31) / 32) * ((g.n[1] + 7) / 8) * ((g.n[2] + kStepZ - 1) / kStepZ);
}

// The step's grid: 32 x 8 columns, and along z blocks of a.zchunk step tiles.
static dim3 step_grid(fw_ctx* ctx, InvArgs& a) {
    const long long gx = (a.g.nx + 31) / 32, gy = (a.g.ny + 7) / 8;
    const long long gz = (a.g.nz + kStepZ - 1) / kStepZ;
    const int64_t n[3] = {a.g.nx, a.g.ny, a.g.nz};
    a.zchunk = inv_step_zchunk(n, ctx->num_sms);
    return dim3((unsigned int)gx, (unsigned int)gy, (unsigned int)((gz + a.zchunk - 1) / a.zchunk));
}

// Scratch of a body: the step's block partials (two doubles a block, at most one block a tile),
// then its deferred list (one entry a warp part: 32 columns of a row, kStepZ slices).
static unsigned int* defer_list(fw_ctx* ctx, const HostGrid& g) {
    return reinterpret_cast<unsigned int*>(ctx->d_scratch + SLOT_PARTIALS + 2 * inv_step_tiles(g));
}

// Before the loop: scratch for its bodies and the loop's settings (the init kernel also sets the
// WHILE node's condition in graph mode).
int enqueue_inversion_prefix(fw_ctx* ctx, const fw_field* field, fw_field* inverse,
                             fw_field* res, const fw_invert_params& prm, InvState* st,
                             cudaGraphConditionalHandle handle, int use_handle) {
    FW_CHECK(res->grid.same(inverse->grid) && res->ps == inverse->ps,
             "invert: the residual buffer does not match the inverse");
    FW_TRY(ensure_scratch(ctx, inv_scratch_doubles(field->grid)));
    k_inv_init<<<1, 1, 0, ctx->stream>>>(st, prm, handle, use_handle);
    return check_launch(ctx, "k_inv_init");
}

// Scratch for the bodies of an inversion of `field` (before a capture: the graph holds the
// pointers).
int inversion_scratch(fw_ctx* ctx, const fw_field* field) {
    return ensure_scratch(ctx, inv_scratch_doubles(field->grid));
}

int enqueue_inversion_inits(fw_ctx* ctx, InvState* st, int count, const fw_invert_params& prm,
                            const cudaGraphConditionalHandle* handles, unsigned int* zero,
                            int nzero) {
    FW_CHECK(count >= 0 && count <= kMaxInitHandles && nzero >= 0 && nzero <= 32,
             "inversion inits: too many loops");
    InitHandles hs;
    for (int i = 0; i < kMaxInitHandles; ++i) hs.h[i] = i < count ? handles[i] : 0;
    return launch_pdl(ctx, "k_inv_init_many", k_inv_init_many, dim3(1), dim3(32), 0, st, count,
                      prm, hs, zero, nzero);
}

// One kernel of a body: 0 bound, 1 step, 2 fix (each returns at once when the loop has ended).
static int launch_body_kernel(fw_ctx* ctx, const fw_field* field, fw_field* inverse,
                              fw_field* res, InvState* st, int which,
                              cudaGraphConditionalHandle handle, int use_handle) {
    InvArgs a = inv_args(field, inverse);
    const dim3 g = step_grid(ctx, a);
    unsigned int* defer = defer_list(ctx, field->grid);
    if (which == 0) {
        const Lattice t = lattice_of(a.g);
        const unsigned int nb = (unsigned int)std::max<long long>(
            1, std::min<long long>((t.count() + 255) / 256, 4LL * ctx->num_sms));
        return launch_pdl(ctx, "k_inv_bound", k_inv_bound, dim3(nb), dim3(256), 0, a, t,
                          (const float*)field->d, (const float*)inverse->d, st);
    }
    if (which == 1)
        return launch_pdl(ctx, "k_inv_step", k_inv_step, g, dim3(256), 0, a,
                          (const float*)field->d, inverse->d, res->d,
                          ctx->d_scratch + SLOT_PARTIALS, ctx->d_counter + 2, st, defer, handle,
                          use_handle);
    const unsigned int tiles = (unsigned int)inv_step_tiles(field->grid);
    const unsigned int nf = std::max(1u, std::min(tiles, 2u * (unsigned int)ctx->num_sms));
    return launch_pdl(ctx, "k_inv_fix", k_inv_fix, dim3(nf), dim3(256), 0, a, inverse->d,
                      (const float*)res->d, (const InvState*)st, (const unsigned int*)defer);
}

// One body: bound, step, fix.
int enqueue_inversion_body(fw_ctx* ctx, const fw_field* field, fw_field* inverse, fw_field* res,
                           InvState* st, cudaGraphConditionalHandle handle, int use_handle) {
    for (int which = 0; which < 3; ++which)
        FW_TRY(launch_body_kernel(ctx, field, inverse, res, st, which, handle, use_handle));
    return 0;
}

int enqueue_inversion_kernel(fw_ctx* ctx, const fw_field* field, fw_field* inverse, fw_field* res,
                             InvState* st, int which) {
    return launch_body_kernel(ctx, field, inverse, res, st, which, 0, 0);
}

size_t inv_scratch_doubles(const HostGrid& g) {
    const size_t tiles = (size_t)inv_step_tiles(g), parts = (size_t)inv_step_parts(g);
    return SLOT_PARTIALS + 2 * tiles + (parts + 1) / 2 + 16;
}

long long inv_bound_voxels(const HostGrid& g) {
    return lattice_of(dev_grid(g)).count();
}

static InvArgs inv_args_grid(const HostGrid& g, long long ps) {
    InvArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = dev_grid(g);
    a.ps_f = ps;
    a.ps_psi = ps;
    a.isx = (float)(1.0 / g.sp[0]);
    a.isy = (float)(1.0 / g.sp[1]);
    a.isz = (float)(1.0 / g.sp[2]);
    return a;
}

int inv_step_blocks(const HostGrid& g, int zchunk) {
    const long long gx = (g.n[0] + 31) / 32, gy = (g.n[1] + 7) / 8;
    const long long gz = (g.n[2] + kStepZ - 1) / kStepZ;
    return (int)(gx * gy * ((gz + zchunk - 1) / zchunk));
}

int inv_bound_vblocks(const HostGrid& g) {
    return (int)std::max<long long>(1, (lattice_of(dev_grid(g)).count() + 255) / 256);
}

int launch_inv_init_batch(fw_ctx* ctx, const BatchList& L, InvState* st, int st_stride,
                          const fw_invert_params& prm) {
    k_inv_init_batch<<<1, 256, 0, ctx->stream>>>(L, st, st_stride, prm);
    return check_launch(ctx, "k_inv_init_batch");
}

int launch_inv_body_batch(fw_ctx* ctx, const HostGrid& g, long long ps, const InvBatchBody& w,
                          const float* f, float* psi, float* res, long long stride,
                          double* partials, long long part_stride, unsigned int* counter,
                          InvState* st, int st_stride, unsigned int* defer,
                          long long defer_stride, int which) {
    InvArgs a = inv_args_grid(g, ps);
    a.zchunk = w.zchunk;
    if (which < 0 || which == 0) {
        k_inv_bound_batch<<<w.bound_blocks, 256, 0, ctx->stream>>>(
            a, lattice_of(a.g), w.bound, f, psi, stride, st, st_stride);
        FW_TRY(check_launch(ctx, "k_inv_bound_batch"));
    }
    if (which < 0 || which == 1) {
        k_inv_step_batch<<<w.step_blocks, 256, 0, ctx->stream>>>(
            a, w.step, f, psi, res, stride, partials, part_stride, counter, st, st_stride, defer,
            defer_stride);
        FW_TRY(check_launch(ctx, "k_inv_step_batch"));
    }
    if (which < 0 || which == 2) {
        k_inv_fix_batch<<<w.fix_blocks, 256, 0, ctx->stream>>>(a, w.fix, psi, res, stride, st,
                                                               st_stride, defer, defer_stride);
        FW_TRY(check_launch(ctx, "k_inv_fix_batch"));
    }
    return 0;
}

int launch_inv_any(fw_ctx* ctx, const InvState* st, int st_stride, const BatchList& L,
                   cudaGraphConditionalHandle handle) {
    k_inv_any<<<1, 32, 0, ctx->stream>>>(st, st_stride, L, handle);
    return check_launch(ctx, "k_inv_any");
}

// Host-driven loop (Backend::invert): one read-back of the loop flag per body.
int invert_field(fw_ctx* ctx, const fw_field* field, fw_field* inverse,
                 const fw_invert_params& prm, fw_invert_stats* stats) {
    InvState* st = reinterpret_cast<InvState*>(ctx->d_scratch + SLOT_INV);
    fw_field* res = nullptr;  // the residual of the last measurement
    FW_TRY(new_field(ctx, inverse->grid, &res));
    struct Free {
        fw_field* f;
        ~Free() { fw_field_free(f); }
    } guard{res};
    FW_TRY(enqueue_inversion_prefix(ctx, field, inverse, res, prm, st, 0, 0));
    InvState h;
    for (int body = 0; body < std::max(prm.max_iterations, 0); ++body) {
        FW_TRY(enqueue_inversion_body(ctx, field, inverse, res, st, 0, 0));
        FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, st, sizeof(InvState), cudaMemcpyDeviceToHost,
                                ctx->stream));
        FW_TRY(sync(ctx));
        std::memcpy(&h, ctx->h_pinned, sizeof(h));
        if (!h.go) break;
    }
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, st, sizeof(InvState), cudaMemcpyDeviceToHost,
                            ctx->stream));
    FW_TRY(sync(ctx));
    std::memcpy(&h, ctx->h_pinned, sizeof(h));
    stats->iterations = h.executed;
    stats->mean_error_norm = h.executed == 0 ? 0.0 : h.mean;
    stats->max_error_norm = h.executed == 0 ? 0.0 : h.max;
    return 0;
}

size_t inv_state_bytes() { return sizeof(InvState); }

void inv_state_read(const void* raw, fw_invert_stats* stats) {
    InvState h;
    std::memcpy(&h, raw, sizeof(h));
    stats->iterations = h.executed;
    stats->mean_error_norm = h.executed == 0 ? 0.0 : h.mean;
    stats->max_error_norm = h.executed == 0 ? 0.0 : h.max;
}

}  // namespace fw

using namespace fw;

extern "C" {

int fw_invert(fw_ctx* ctx, const fw_field* field, fw_field* initial,
              const fw_invert_params* params, fw_invert_stats* stats) {
    FW_CHECK(ctx && field && initial && params && stats, "null argument");
    if (!field->grid.same(initial->grid))
        return fail(FW_ERR_INVALID, "invert: initial estimate grid differs");
    return invert_field(ctx, field, initial, *params, stats);
}

int fw_invert_pair(fw_ctx* ctx, fw_field* field, fw_field* inverse,
                   const fw_invert_params* params, fw_invert_stats stats[2]) {
    FW_CHECK(ctx && field && inverse && params && stats, "null argument");
    if (!field->grid.same(inverse->grid))
        return fail(FW_ERR_INVALID, "invert: initial estimate grid differs");
    FW_TRY(invert_field(ctx, field, inverse, *params, &stats[0]));
    return invert_field(ctx, inverse, field, *params, &stats[1]);
}

}  // extern "C"
