// fw_invert.cu -- ITK InvertDisplacementFieldImageFilter as SyN runs it (field_ops.rs:309-392).
//
// The reference loop is: while (iteration < max && max_error > max_tol && mean_error > mean_tol)
// { e = psi + f(x + psi); measure mean and max of |e/sp|; psi += eps * clamp(-e) with
// eps = 0.75 on the first body and 0.5 after; faces of psi to zero }.
//
// Device design: the error at voxel x depends only on psi(x) and the read-only field f, so one
// sweep can apply body k's update to psi(x) and at once measure body k+1's error at the same
// voxel. Each body is therefore ONE sweep (read psi and the kept residual, write psi, gather f
// for the next measurement only when there is a next body) plus a fixed-order reduction done by
// the last block to finish; it is launched as a pair of kernels of which one works. The loop
// state (errors of the last measurement, body index, whether the next body runs) lives in device
// memory and is updated by that last block, so the loop needs no host read-back: the SyN driver
// runs it inside a CUDA graph WHILE node whose condition the last block sets.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>

#include "fw_internal.cuh"

namespace fw {

struct InvArgs {
    DevGrid g;
    long long ps_f, ps_psi;
    float isx, isy, isz;
    int zchunk;  // slices a thread marches through
};

__device__ __forceinline__ void residual(const InvArgs& a, const float* __restrict__ f,
                                         long long l, int i, int j, int k, float px, float py,
                                         float pz, float e[3]) {
    double c0 = i + (a.g.inv[0] * px + a.g.inv[1] * py + a.g.inv[2] * pz);
    double c1 = j + (a.g.inv[3] * px + a.g.inv[4] * py + a.g.inv[5] * pz);
    double c2 = k + (a.g.inv[6] * px + a.g.inv[7] * py + a.g.inv[8] * pz);
    float d[3] = {0.0f, 0.0f, 0.0f};
    if (inside_index(c0, c1, c2, a.g.nx, a.g.ny, a.g.nz))
        vec_at_index(f, a.ps_f, a.g.nx, a.g.ny, a.g.nz, c0, c1, c2, d);
    e[0] = px + d[0];
    e[1] = py + d[1];
    e[2] = pz + d[2];
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

// The measurement of tile (bx, by, bz): the thread's column of e = psi + f(x + psi) kept in
// `res`, its sum and max of |e/sp| added to sum / mx.
__device__ __forceinline__ void measure_tile(const InvArgs& a, int bx, int by, int bz,
                                             const float* __restrict__ f,
                                             const float* __restrict__ psi,
                                             float* __restrict__ res, double& sum, float& mx) {
    struct {
        int x, y, z0, z1;
    } col;
    if (!column_of_tile(a.g.nx, a.g.ny, a.g.nz, a.zchunk, bx, by, bz, col.x, col.y, col.z0,
                        col.z1))
        return;
    const long long sxy = (long long)a.g.nx * a.g.ny;
    long long l = (long long)col.z0 * sxy + (long long)col.y * a.g.nx + col.x;
    float px = psi[l], py = psi[l + a.ps_psi], pz = psi[l + 2 * a.ps_psi];
    for (int z = col.z0; z < col.z1; ++z, l += sxy) {
        float qx = 0.0f, qy = 0.0f, qz = 0.0f;
        if (z + 1 < col.z1) {  // the next slice's psi, in flight during this gather
            qx = psi[l + sxy];
            qy = psi[l + sxy + a.ps_psi];
            qz = psi[l + sxy + 2 * a.ps_psi];
        }
        float e[3];
        residual(a, f, l, col.x, col.y, z, px, py, pz, e);
        res[l] = e[0];
        res[l + a.ps_psi] = e[1];
        res[l + 2 * a.ps_psi] = e[2];
        float x = e[0] * a.isx, y = e[1] * a.isy, zz = e[2] * a.isz;
        float nrm = nan_canon(sqrtf(x * x + y * y + zz * zz));
        sum += (double)nrm;
        mx = __int_as_float(max(__float_as_int(mx), __float_as_int(nrm)));
        px = qx;
        py = qy;
        pz = qz;
    }
}

// First measurement (body 0's error) of psi against f; the residual e = psi + f(x + psi) of
// every voxel is kept in `res` for the body that follows.
// Its last block also writes the loop's settings into the state (no separate init launch).
__global__ void __launch_bounds__(256, 4) k_inv_measure(InvArgs a, const float* __restrict__ f,
                                                     const float* __restrict__ psi,
                                                     float* __restrict__ res,
                                                     double* __restrict__ partials,
                                                     unsigned int* __restrict__ counter,
                                                     InvState* __restrict__ st,
                                                     fw_invert_params prm,
                                                     cudaGraphConditionalHandle handle,
                                                     int use_handle) {
    double sum = 0.0;
    float mx = 0.0f;
    measure_tile(a, blockIdx.x, blockIdx.y, blockIdx.z, f, psi, res, sum, mx);
    const double count = (double)a.g.n;
    const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const unsigned int nblocks = gridDim.x * gridDim.y * gridDim.z;
    reduce_and_finish(sum, mx, partials, counter, bid, nblocks, [&](double s, double m) {
        st->max_iterations = prm.max_iterations;
        st->mean_tol = prm.mean_error_tolerance;
        st->max_tol = prm.max_error_tolerance;
        st->enforce = prm.enforce_boundary_condition;
        st->mean = s / count;
        st->max = m;
        st->executed = 0;
        st->k = 0;
        st->go = prm.max_iterations > 0 ? 1 : 0;
        if (use_handle) cudaGraphSetConditional(handle, st->go ? 1u : 0u);
    });
}

// The sweep of virtual block vb of nvb (a grid-stride loop over the voxels, two a step): the
// update of psi with eps and limit from the kept residual, faces to zero with `enforce`, and with
// GATHER the next measurement into res, its sum and max added to sum / mx.
template <bool GATHER>
__device__ __forceinline__ void body_sweep(const InvArgs& a, unsigned int vb, unsigned int nvb,
                                           const float* __restrict__ f, float* __restrict__ psi,
                                           float* __restrict__ res, float eps, float limit,
                                           bool enforce, double& sum, float& mx) {
    const long long stride = (long long)nvb * blockDim.x;
    // two voxels a step, `stride` apart: their loads are in flight together
    for (long long l0 = (long long)vb * blockDim.x + threadIdx.x; l0 < a.g.n;
         l0 += 2 * stride) {
        float px[2], py[2], pz[2], ex[2], ey[2], ez[2];
        int ii[2], jj[2], kk[2];
        bool ok[2];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            long long l = l0 + v * stride;
            ok[v] = l < a.g.n;
            if (!ok[v]) continue;
            voxel_ijk(l, a.g.nx, a.g.ny, ii[v], jj[v], kk[v]);
            px[v] = psi[l];
            py[v] = psi[l + a.ps_psi];
            pz[v] = psi[l + 2 * a.ps_psi];
            ex[v] = res[l];
            ey[v] = res[l + a.ps_psi];
            ez[v] = res[l + 2 * a.ps_psi];
        }
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            if (!ok[v]) continue;
            long long l = l0 + v * stride;
            const int i = ii[v], j = jj[v], k = kk[v];
            float sx = ex[v] * a.isx, sy = ey[v] * a.isy, sz = ez[v] * a.isz;
            float nrm = sqrtf(sx * sx + sy * sy + sz * sz);
            float ux = -ex[v], uy = -ey[v], uz = -ez[v];
            if (nrm > limit) {
                float fct = limit / nrm;
                ux *= fct;
                uy *= fct;
                uz *= fct;
            }
            px[v] = px[v] + ux * eps;
            py[v] = py[v] + uy * eps;
            pz[v] = pz[v] + uz * eps;
            const bool face = i == 0 || j == 0 || k == 0 || i == a.g.nx - 1 ||
                              j == a.g.ny - 1 || k == a.g.nz - 1;
            if (enforce && face) px[v] = py[v] = pz[v] = 0.0f;
            psi[l] = px[v];
            psi[l + a.ps_psi] = py[v];
            psi[l + 2 * a.ps_psi] = pz[v];
        }
        if constexpr (GATHER) {
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                if (!ok[v]) continue;
                long long l = l0 + v * stride;
                float e[3];
                residual(a, f, l, ii[v], jj[v], kk[v], px[v], py[v], pz[v], e);
                res[l] = e[0];
                res[l + a.ps_psi] = e[1];
                res[l + 2 * a.ps_psi] = e[2];
                float x = e[0] * a.isx, y = e[1] * a.isy, z = e[2] * a.isz;
                float n2 = nan_canon(sqrtf(x * x + y * y + z * z));
                sum += (double)n2;
                mx = __int_as_float(max(__float_as_int(mx), __float_as_int(n2)));
            }
        }
    }
}

// One body: the update with eps (0.75 on body 0, else 0.5) and limit eps * max of the last
// measurement, from the residual that measurement kept in `res`; faces to zero; then -- when
// the next body will run -- its measurement, whose residual replaces the voxel's in `res`.
// Two kernels share the work, launched in this order every body: GATHER = false runs the body
// when the loop stops after it (an elementwise sweep, no gather), GATHER = true when the loop
// goes on (update and next measurement in one sweep). Each decides from the loop state, which
// only the kernel that runs changes (in its last block), so exactly one of them works; kept
// apart, the elementwise sweep keeps the gather's register footprint out of its occupancy.
template <bool GATHER>
__global__ void __launch_bounds__(256, 4) k_inv_body(InvArgs a, const float* __restrict__ f,
                                                     float* __restrict__ psi,
                                                     float* __restrict__ res,
                                                     double* __restrict__ partials,
                                                     unsigned int* __restrict__ counter,
                                                     InvState* __restrict__ st,
                                                     cudaGraphConditionalHandle handle,
                                                     int use_handle) {
    const int go = st->go;
    if (!go) {  // uniform: the state only changes in the last block of the grid that works
        // keep a WHILE loop from spinning should its condition ever disagree with the state
        if (use_handle && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(handle, 0u);
        return;
    }
    const int kb = st->k;
    const double mean = st->mean, mxe = st->max;
    const bool next = (kb + 1 < st->max_iterations) && mxe > st->max_tol && mean > st->mean_tol;
    if (next != GATHER) return;  // the other kernel of the pair runs this body
    const float eps = kb == 0 ? 0.75f : 0.5f;
    const float limit = eps * (float)mxe;
    const bool enforce = st->enforce != 0;
    double sum = 0.0;
    float mx = 0.0f;
    body_sweep<GATHER>(a, blockIdx.x, gridDim.x, f, psi, res, eps, limit, enforce, sum, mx);
    const double count = (double)a.g.n;
    reduce_and_finish(sum, mx, partials, counter, blockIdx.x, gridDim.x, [&](double s, double m) {
        st->executed = kb + 1;
        if (GATHER) {
            st->mean = s / count;
            st->max = m;
            st->k = kb + 1;
        }
        st->go = GATHER ? 1 : 0;
        if (use_handle) cudaGraphSetConditional(handle, GATHER ? 1u : 0u);
    });
}

// ---- batched inversions: every active subject of a batch, each with its own loop state ------
//
// Subject b's field, inverse and residual are at f / psi / res + b * stride, its partials at
// partials + b * part_stride, its last-item counter at counter[b] and its loop state at
// st[b * st_stride]. Tiles and virtual blocks are those of the single kernels, and a subject's
// partials are reduced in the same order, so its loop takes the same decisions as alone. The
// loop's condition is set afterwards by k_inv_any (any active subject still iterating).

__global__ void __launch_bounds__(256, 4) k_inv_measure_batch(
    InvArgs a, BatchList L, const float* __restrict__ f, const float* __restrict__ psi,
    float* __restrict__ res, long long stride, double* __restrict__ partials,
    long long part_stride, unsigned int* __restrict__ counter, InvState* __restrict__ st,
    int st_stride, fw_invert_params prm) {
    const int work = *L.count * L.tiles;
    const int gx = (a.g.nx + 31) / 32, gy = (a.g.ny + 7) / 8;
    const double count = (double)a.g.n;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles], t = w % L.tiles;
        int bx, by, bz;
        tile_coords(t, gx, gy, bx, by, bz);
        double sum = 0.0;
        float mx = 0.0f;
        measure_tile(a, bx, by, bz, f + b * stride, psi + b * stride, res + b * stride, sum, mx);
        InvState* sb = st + b * st_stride;
        reduce_and_finish(sum, mx, partials + b * part_stride, counter + b, (unsigned int)t,
                          (unsigned int)L.tiles, [&](double sm, double m) {
                              sb->max_iterations = prm.max_iterations;
                              sb->mean_tol = prm.mean_error_tolerance;
                              sb->max_tol = prm.max_error_tolerance;
                              sb->enforce = prm.enforce_boundary_condition;
                              sb->mean = sm / count;
                              sb->max = m;
                              sb->executed = 0;
                              sb->k = 0;
                              sb->go = prm.max_iterations > 0 ? 1 : 0;
                          });
        __syncthreads();  // the next item reuses the reduction's shared memory
    }
}

// One body of every active subject (virtual block vb of L.tiles per subject): the kernel of the
// pair that matches the subject's next step works, the other skips the subject.
template <bool GATHER>
__global__ void __launch_bounds__(256, 4) k_inv_body_batch(
    InvArgs a, BatchList L, const float* __restrict__ f, float* __restrict__ psi,
    float* __restrict__ res, long long stride, double* __restrict__ partials,
    long long part_stride, unsigned int* __restrict__ counter, InvState* __restrict__ st,
    int st_stride) {
    const int work = *L.count * L.tiles;
    const double count = (double)a.g.n;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles];
        const unsigned int vb = (unsigned int)(w % L.tiles);
        InvState* sb = st + b * st_stride;
        // uniform over the block; the state only changes once every item of the subject is done
        if (!sb->go) continue;
        const int kb = sb->k;
        const double mean = sb->mean, mxe = sb->max;
        const bool next = (kb + 1 < sb->max_iterations) && mxe > sb->max_tol && mean > sb->mean_tol;
        if (next != GATHER) continue;
        const float eps = kb == 0 ? 0.75f : 0.5f;
        const float limit = eps * (float)mxe;
        double sum = 0.0;
        float mx = 0.0f;
        body_sweep<GATHER>(a, vb, (unsigned int)L.tiles, f + b * stride, psi + b * stride,
                           res + b * stride, eps, limit, sb->enforce != 0, sum, mx);
        reduce_and_finish(sum, mx, partials + b * part_stride, counter + b, vb,
                          (unsigned int)L.tiles, [&](double sm, double m) {
                              sb->executed = kb + 1;
                              if (GATHER) {
                                  sb->mean = sm / count;
                                  sb->max = m;
                                  sb->k = kb + 1;
                              }
                              sb->go = GATHER ? 1 : 0;
                          });
        __syncthreads();
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

// Re-arms a finished loop for one more body from its last measurement (kernel timing).
__global__ void k_inv_rearm(InvState* st, int max_iterations) {
    st->go = 1;
    st->k = 0;
    st->max_iterations = max_iterations;
}

int enqueue_inversion_rearm(fw_ctx* ctx, InvState* st, int max_iterations) {
    k_inv_rearm<<<1, 1, 0, ctx->stream>>>(st, max_iterations);
    return check_launch(ctx, "k_inv_rearm");
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

// The body streams psi and the residual (a flat grid-stride sweep, two voxels a step); only when
// the loop goes on does it gather, and the measurement -- a gather of every voxel -- runs over
// 32 x 8 column tiles marching along z (z chunks so that the grid fills the GPU a few blocks
// deep per SM).
// One wave of resident blocks (the body kernels keep 4 blocks of 256 threads on an SM; the sweep
// loops over the rest): the kernel of a body pair that returns at once costs half as much as
// with two waves, and the working one is as fast or faster.
static unsigned int inv_blocks(fw_ctx* ctx, long long n) {
    long long b = (n + 255) / 256;
    return (unsigned int)std::max<long long>(1, std::min<long long>(b, 4LL * ctx->num_sms));
}

static dim3 inv_grid(fw_ctx* ctx, InvArgs& a) {
    return column_grid(a.g.nx, a.g.ny, a.g.nz, ctx->num_sms, &a.zchunk);
}

// Launches the whole inversion on the stream: init, first measurement and `bodies` body kernels
// (each returns at once after the loop has ended). Used by graph capture with bodies = 0.
int enqueue_inversion_prefix(fw_ctx* ctx, const fw_field* field, fw_field* inverse,
                             fw_field* res, const fw_invert_params& prm, InvState* st,
                             cudaGraphConditionalHandle handle, int use_handle) {
    FW_CHECK(res->grid.same(inverse->grid) && res->ps == inverse->ps,
             "invert: the residual buffer does not match the inverse");
    InvArgs a = inv_args(field, inverse);
    const dim3 blocks = inv_grid(ctx, a);
    // block partials of the measurement's tiles and of the bodies' flat grid
    const size_t parts = std::max<size_t>((size_t)blocks.x * blocks.y * blocks.z,
                                          inv_blocks(ctx, a.g.n));
    FW_TRY(ensure_scratch(ctx, SLOT_PARTIALS + 2 * parts + 16));
    k_inv_measure<<<blocks, 256, 0, ctx->stream>>>(a, field->d, inverse->d, res->d,
                                                   ctx->d_scratch + SLOT_PARTIALS,
                                                   ctx->d_counter + 2, st, prm, handle, use_handle);
    return check_launch(ctx, "k_inv_measure");
}

int enqueue_inversion_body(fw_ctx* ctx, const fw_field* field, fw_field* inverse, fw_field* res,
                           InvState* st, cudaGraphConditionalHandle handle, int use_handle) {
    InvArgs a = inv_args(field, inverse);
    const unsigned int blocks = inv_blocks(ctx, a.g.n);
    k_inv_body<false><<<blocks, 256, 0, ctx->stream>>>(a, field->d, inverse->d, res->d,
                                                       ctx->d_scratch + SLOT_PARTIALS,
                                                       ctx->d_counter + 2, st, handle, use_handle);
    FW_TRY(check_launch(ctx, "k_inv_body"));
    k_inv_body<true><<<blocks, 256, 0, ctx->stream>>>(a, field->d, inverse->d, res->d,
                                                      ctx->d_scratch + SLOT_PARTIALS,
                                                      ctx->d_counter + 2, st, handle, use_handle);
    return check_launch(ctx, "k_inv_body");
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

int inv_measure_tiles(const HostGrid& g, int zchunk) {
    const long long gx = (g.n[0] + 31) / 32, gy = (g.n[1] + 7) / 8, gz = (g.n[2] + zchunk - 1) / zchunk;
    return (int)(gx * gy * gz);
}

int inv_body_vblocks(fw_ctx* ctx, long long n) { return (int)inv_blocks(ctx, n); }

int launch_inv_measure_batch(fw_ctx* ctx, const HostGrid& g, long long ps, int zchunk,
                             const BatchList& L, int blocks, const float* f, const float* psi,
                             float* res, long long stride, double* partials,
                             long long part_stride, unsigned int* counter, InvState* st,
                             int st_stride, const fw_invert_params& prm) {
    InvArgs a = inv_args_grid(g, ps);
    a.zchunk = zchunk;
    k_inv_measure_batch<<<blocks, 256, 0, ctx->stream>>>(a, L, f, psi, res, stride, partials,
                                                         part_stride, counter, st, st_stride, prm);
    return check_launch(ctx, "k_inv_measure_batch");
}

int launch_inv_body_batch(fw_ctx* ctx, const HostGrid& g, long long ps, const BatchList& L,
                          int blocks, const float* f, float* psi, float* res, long long stride,
                          double* partials, long long part_stride, unsigned int* counter,
                          InvState* st, int st_stride) {
    InvArgs a = inv_args_grid(g, ps);
    k_inv_body_batch<false><<<blocks, 256, 0, ctx->stream>>>(a, L, f, psi, res, stride, partials,
                                                             part_stride, counter, st, st_stride);
    FW_TRY(check_launch(ctx, "k_inv_body_batch"));
    k_inv_body_batch<true><<<blocks, 256, 0, ctx->stream>>>(a, L, f, psi, res, stride, partials,
                                                            part_stride, counter, st, st_stride);
    return check_launch(ctx, "k_inv_body_batch");
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
