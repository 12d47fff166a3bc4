// fw_internal.cuh -- shared declarations of the sm_100a registration engine.
//
// Device layout: images are float32 arrays of n = nx*ny*nz voxels (x fastest); fields are three
// float32 planes (x | y | z) of `ps` floats each, ps = n rounded up to 64 so every plane starts
// on a 256-byte boundary and 16-byte vector accesses stay aligned.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cmath>
#include <mutex>
#include <string>
#include <chrono>
#include <future>
#include <list>
#include <unordered_map>
#include <vector>

#include "../../include/fastwarp_cuda.h"

namespace fw {

// ---- errors ---------------------------------------------------------------------------------

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define FW_CUDA(call)                                              \
    do {                                                           \
        cudaError_t fw_e_ = (call);                                \
        if (fw_e_ != cudaSuccess) return ::fw::cuda_fail(fw_e_, #call); \
    } while (0)

#define FW_CHECK(cond, msg)                                        \
    do {                                                           \
        if (!(cond)) return ::fw::fail(FW_ERR_INVALID, (msg));     \
    } while (0)

#define FW_TRY(call)                  \
    do {                              \
        int fw_rc_ = (call);          \
        if (fw_rc_ != 0) return fw_rc_; \
    } while (0)

// ---- host grid math (grid.rs:45-161) -------------------------------------------------------

struct HostGrid {
    int64_t n[3];
    double sp[3], org[3], dir[9];
    double ds[9];   // direction * diag(spacing): index -> offset
    double inv[9];  // its inverse: offset -> index
    int64_t count() const { return n[0] * n[1] * n[2]; }
    bool same(const HostGrid& o) const;
};

bool mat3_inverse(const double m[9], double out[9]);
void mat3_mul(const double a[9], const double b[9], double out[9]);
void mat3_vec(const double m[9], const double v[3], double out[3]);
int make_grid(const fw_grid* g, HostGrid& out);
fw_grid to_c(const HostGrid& g);

// ---- device grid ---------------------------------------------------------------------------

struct DevGrid {
    int nx, ny, nz;
    long long n;
    double org[3];
    double ds[9];
    double inv[9];
    double sp[3];
    double dir[9];
};

DevGrid dev_grid(const HostGrid& g);

inline int64_t plane_stride(int64_t n) { return (n + 63) / 64 * 64; }

// ---- context and buffers -------------------------------------------------------------------

}  // namespace fw

struct fw_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    // scratch: reduction partials, small device scalars and a pinned host mirror
    double* d_scratch = nullptr;     // device scratch doubles
    size_t scratch_doubles = 0;
    unsigned int* d_counter = nullptr;  // last-block counters (zeroed after use)
    double* h_pinned = nullptr;      // pinned host scalars for read-backs
    void* h_stage = nullptr;         // pinned host staging for larger uploads (grown on demand)
    size_t h_stage_bytes = 0;
    fw_stats stats{};
    std::atomic<uint64_t> live_bytes{0};
    const volatile int32_t* cancel = nullptr;  // the caller's flag (fw_ctx_set_cancel_flag)
    // the context's own flag (fw_ctx_request_cancel) in mapped pinned host memory: the host view
    // and the device view, which the level graph's record kernel reads once per iteration
    volatile int32_t* cancel_mapped = nullptr;
    const volatile int32_t* cancel_mapped_dev = nullptr;
    bool capturing = false;          // a graph capture is in progress on `stream`
    cudaStream_t aux = nullptr;      // second stream for capturing conditional bodies
    cudaEvent_t done = nullptr;      // blocking-sync event the host waits on
    cudaMemPool_t pool = nullptr;    // the context's own stream-ordered memory pool
    // freed buffers kept by size for the next allocation of that size (stream order makes the
    // reuse safe: every user of a buffer runs on `stream`); guarded for frees from other threads.
    // `cache_lru` holds them in the order they were freed, `cache` indexes it by size.
    struct CachedBuffer {
        size_t size;
        void* p;
        std::chrono::steady_clock::time_point freed;
    };
    std::mutex cache_mu;
    std::list<CachedBuffer> cache_lru;
    // the regular sampler's generator integers on the device, kept by (seed, picks) for the next
    // registration of the same level grid (a few buffers, the least recently used out first);
    // used by the context's own thread only
    struct DrawBuffer {
        uint32_t seed;
        int64_t picks;
        uint32_t* d;
        size_t bytes;
        uint64_t used;
    };
    std::vector<DrawBuffer> draws;
    uint64_t draws_tick = 0;
    std::unordered_multimap<size_t, std::list<CachedBuffer>::iterator> cache;
    uint64_t cached_bytes = 0;
};

struct fw_image {
    fw_ctx* ctx;
    fw::HostGrid grid;
    float* d;
    size_t bytes;
};

struct fw_field {
    fw_ctx* ctx;
    fw::HostGrid grid;
    float* d;       // plane 0; planes at d, d + ps, d + 2 ps
    int64_t ps;     // plane stride in floats
    size_t bytes;
};

namespace fw {

// Whether a cancel has been asked for, through the caller's flag or the context's own.
inline bool cancel_requested(const fw_ctx* ctx) {
    return (ctx->cancel && *ctx->cancel) || (ctx->cancel_mapped && *ctx->cancel_mapped);
}

// stream-ordered allocation from the device's memory pool (kept cached: the buffer pool)
int dev_alloc(fw_ctx* ctx, size_t bytes, void** out);
void dev_free(fw_ctx* ctx, void* p, size_t bytes);
int new_image(fw_ctx* ctx, const HostGrid& g, fw_image** out);
int new_field(fw_ctx* ctx, const HostGrid& g, fw_field** out);
int sync(fw_ctx* ctx);
int check_launch(fw_ctx* ctx, const char* what);

// Programmatic dependent launch (sm_90+): a kernel launched by launch_pdl may be scheduled while
// the kernel before it on the stream drains, so the launch latency of a chain of small kernels
// (the coarse pyramid levels) overlaps the previous kernel's tail. Every such kernel calls
// pdl_wait() before its first memory access: it returns once the previous kernel has completed
// and its writes are visible, so the kernel sees exactly what an ordinary launch would (for an
// ordinary launch it returns at once). FASTWARP_PDL=0 launches them without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
bool pdl_enabled();

template <typename... KArgs, typename... Args>
int launch_pdl(fw_ctx* ctx, const char* what, void (*kernel)(KArgs...), dim3 grid, dim3 block,
               size_t smem, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
    if (e != cudaSuccess) return cuda_fail(e, what);
    return check_launch(ctx, what);
}
// The context's pinned staging buffer, at least `bytes` long; the caller synchronises the
// stream before it writes the buffer again.
int host_stage(fw_ctx* ctx, size_t bytes, void** out);
int ensure_scratch(fw_ctx* ctx, size_t doubles);

// ---- device helpers: ITK interpolation rules (interp.rs:43-120, field_ops.rs:143-181) -----

// ITK IsInsideBuffer on a continuous index: every coordinate in [-0.5, n - 0.5).
__device__ __forceinline__ bool inside_index(double cx, double cy, double cz, int nx, int ny,
                                             int nz) {
    return cx >= -0.5 && cx < (double)nx - 0.5 && cy >= -0.5 && cy < (double)ny - 0.5 &&
           cz >= -0.5 && cz < (double)nz - 0.5;
}

// One axis of ITK's scalar linear interpolation: base clamped into the buffer, no weight when
// the distance is not positive or the upper neighbour is past the last voxel.
// The three cases keep the f64 subtraction of the clamped base exact without converting the base
// back to f64 (one conversion fewer per axis).
__device__ __forceinline__ void lin_axis(double c, int n, int& b, float& w) {
    const double fl = floor(c);
    double d;
    if (fl < 0.0) {  // clamped to the first voxel
        b = 0;
        d = c;
    } else if (!(fl <= (double)(n - 1))) {  // clamped to the last (NaN too)
        b = n - 1;
        d = c - (double)(n - 1);
    } else {
        b = (int)fl;
        d = c - fl;
    }
    w = (d <= 0.0 || b + 1 > n - 1) ? 0.0f : (float)d;
}

// interp.rs:43-85: LinearInterpolateImageFunction::EvaluateAtContinuousIndex (no bounds check).
// Voxel offsets are 32-bit (grids hold fewer than 2^31 voxels).
__device__ __forceinline__ float lin_at_index(const float* __restrict__ img, int nx, int ny,
                                              int nz, double cx, double cy, double cz) {
    int bx, by, bz;
    float wx, wy, wz;
    lin_axis(cx, nx, bx, wx);
    lin_axis(cy, ny, by, wy);
    lin_axis(cz, nz, bz, wz);
    const unsigned int sy = (unsigned int)nx, sz = (unsigned int)nx * (unsigned int)ny;
    const unsigned int b = (unsigned int)bx + sy * (unsigned int)by + sz * (unsigned int)bz;
    const unsigned int ox = wx > 0.0f ? 1u : 0u;
    const unsigned int oy = wy > 0.0f ? sy : 0u;
    const unsigned int oz = wz > 0.0f ? sz : 0u;
    float v000 = __ldg(img + b), v100 = __ldg(img + (b + ox));
    float v010 = __ldg(img + (b + oy)), v110 = __ldg(img + (b + oy + ox));
    float x0 = fmaf(v100 - v000, wx, v000);
    float x1 = fmaf(v110 - v010, wx, v010);
    float y0 = fmaf(x1 - x0, wy, x0);
    if (wz > 0.0f) {
        float v001 = __ldg(img + (b + oz)), v101 = __ldg(img + (b + oz + ox));
        float v011 = __ldg(img + (b + oz + oy)), v111 = __ldg(img + (b + oz + oy + ox));
        float x2 = fmaf(v101 - v001, wx, v001);
        float x3 = fmaf(v111 - v011, wx, v011);
        float y1 = fmaf(x3 - x2, wy, x2);
        return fmaf(y1 - y0, wz, y0);
    }
    return y0;
}

// field_ops.rs:143-172: VectorLinearInterpolateImageFunction (neighbours clamped, weights 1-d, d)
// of a SoA field at a continuous index. The eight corner weights are formed once for the three
// planes; voxel offsets are 32-bit (grids hold fewer than 2^31 voxels). A corner of weight zero
// adds nothing, as in the reference, by a select rather than a branch, so that all 24 loads can
// be in flight at once (every corner address is inside the buffer: the indices are clamped).
__device__ __forceinline__ void vec_at_index(const float* __restrict__ f, long long ps, int nx,
                                             int ny, int nz, double cx, double cy, double cz,
                                             float out[3]) {
    double fx = floor(cx), fy = floor(cy), fz = floor(cz);
    float dx = (float)(cx - fx), dy = (float)(cy - fy), dz = (float)(cz - fz);
    int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
    int xa = min(max(x0, 0), nx - 1), xb = min(max(x0 + 1, 0), nx - 1);
    int ya = min(max(y0, 0), ny - 1), yb = min(max(y0 + 1, 0), ny - 1);
    int za = min(max(z0, 0), nz - 1), zb = min(max(z0 + 1, 0), nz - 1);
    const unsigned int sy = (unsigned int)nx, sz = (unsigned int)nx * (unsigned int)ny;
    const unsigned int b = (unsigned int)xa + sy * (unsigned int)ya + sz * (unsigned int)za;
    const unsigned int ox = (unsigned int)(xb - xa), oy = sy * (unsigned int)(yb - ya),
                       oz = sz * (unsigned int)(zb - za);
    const unsigned int off[8] = {b, b + ox, b + oy, b + oy + ox,
                                 b + oz, b + oz + ox, b + oz + oy, b + oz + oy + ox};
    const float w0[3] = {1.0f - dx, 1.0f - dy, 1.0f - dz}, w1[3] = {dx, dy, dz};
    const float o[8] = {w0[0] * w0[1] * w0[2], w1[0] * w0[1] * w0[2], w0[0] * w1[1] * w0[2],
                        w1[0] * w1[1] * w0[2], w0[0] * w0[1] * w1[2], w1[0] * w0[1] * w1[2],
                        w0[0] * w1[1] * w1[2], w1[0] * w1[1] * w1[2]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float* p = f + c * ps;
        float acc = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float v = __ldg(p + off[q]);
            acc = o[q] != 0.0f ? fmaf(o[q], v, acc) : acc;
        }
        out[c] = acc;
    }
}

// Grid::index_to_point then another grid's Grid::point_to_index (grid.rs:131-156) in the
// reference's float64 operation order with no fused multiply-adds, so points on a buffer edge
// (-0.5 or n - 0.5) fall on the same side as in the reference.
__device__ __forceinline__ void exact_point(const DevGrid& g, double i, double j, double k,
                                            double p[3]) {
    double s0 = __dmul_rn(i, g.sp[0]), s1 = __dmul_rn(j, g.sp[1]), s2 = __dmul_rn(k, g.sp[2]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
        p[r] = __dadd_rn(g.org[r], __dadd_rn(__dadd_rn(__dmul_rn(g.dir[r * 3], s0),
                                                       __dmul_rn(g.dir[r * 3 + 1], s1)),
                                             __dmul_rn(g.dir[r * 3 + 2], s2)));
}

__device__ __forceinline__ void exact_index(const DevGrid& g, const double p[3], double c[3]) {
    double e0 = __dsub_rn(p[0], g.org[0]), e1 = __dsub_rn(p[1], g.org[1]),
           e2 = __dsub_rn(p[2], g.org[2]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
        c[r] = __dadd_rn(__dadd_rn(__dmul_rn(g.inv[r * 3], e0), __dmul_rn(g.inv[r * 3 + 1], e1)),
                         __dmul_rn(g.inv[r * 3 + 2], e2));
}

// Exact float64 emulation of the oracle's probe position (index_to_point, offset along the
// physical axis, point_to_index) -- no fused multiply-adds, so the inside test at the faces
// rounds as the reference's f64 code does.
__device__ __forceinline__ void probe_index(const DevGrid& g, int i, int j, int k, int d,
                                            double sign, double c[3]) {
    double s0 = __dmul_rn((double)i, g.sp[0]);
    double s1 = __dmul_rn((double)j, g.sp[1]);
    double s2 = __dmul_rn((double)k, g.sp[2]);
    double p[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double rot = __dadd_rn(__dadd_rn(__dmul_rn(g.dir[r * 3 + 0], s0),
                                         __dmul_rn(g.dir[r * 3 + 1], s1)),
                               __dmul_rn(g.dir[r * 3 + 2], s2));
        p[r] = __dadd_rn(g.org[r], rot);
    }
    double off = __dmul_rn(0.5, g.sp[d]);
    p[d] = sign > 0 ? __dadd_rn(p[d], off) : __dsub_rn(p[d], off);
    double e0 = __dsub_rn(p[0], g.org[0]), e1 = __dsub_rn(p[1], g.org[1]),
           e2 = __dsub_rn(p[2], g.org[2]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
        c[r] = __dadd_rn(__dadd_rn(__dmul_rn(g.inv[r * 3], e0), __dmul_rn(g.inv[r * 3 + 1], e1)),
                         __dmul_rn(g.inv[r * 3 + 2], e2));
}

// interp.rs:96-120 at voxel (i, j, k) from global memory, general direction.
__device__ __forceinline__ void central_difference_exact(const float* __restrict__ img,
                                                         const DevGrid& g, int i, int j, int k,
                                                         float out[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double c1[3], c2[3];
        probe_index(g, i, j, k, d, -1.0, c1);
        probe_index(g, i, j, k, d, +1.0, c2);
        out[d] = 0.0f;
        if (!inside_index(c1[0], c1[1], c1[2], g.nx, g.ny, g.nz) ||
            !inside_index(c2[0], c2[1], c2[2], g.nx, g.ny, g.nz))
            continue;
        float v1 = lin_at_index(img, g.nx, g.ny, g.nz, c1[0], c1[1], c1[2]);
        float v2 = lin_at_index(img, g.nx, g.ny, g.nz, c2[0], c2[1], c2[2]);
        out[d] = (float)((double)(v2 - v1) / g.sp[d]);
    }
}

// Whether the probe of voxel coordinate `i` (axis d, direction `sign`) is inside the buffer,
// for an identity direction: only the two face voxels can round either way.
__device__ __forceinline__ bool axis_probe_inside(const DevGrid& g, int i, int j, int k, int d,
                                                  double sign, int n) {
    int q = d == 0 ? i : (d == 1 ? j : k);
    if (sign < 0 && q > 0) return true;
    if (sign > 0 && q < n - 1) return true;
    double c[3];
    probe_index(g, i, j, k, d, sign, c);
    return c[d] >= -0.5 && c[d] < (double)n - 0.5;
}

// interp.rs:96-120 at voxel (x, y, z) from global memory. On an identity-direction grid the
// probes at +-half a spacing lerp halfway toward the neighbours along the axis (the face voxels
// decided by the exact probe test); otherwise the exact probes.
__device__ __forceinline__ void central_difference_voxel(const float* __restrict__ img,
                                                         const DevGrid& g, bool identity,
                                                         const double isp[3], int x, int y,
                                                         int z, float out[3]) {
    if (!identity) {
        central_difference_exact(img, g, x, y, z, out);
        return;
    }
    const int nn[3] = {g.nx, g.ny, g.nz};
    const int pos[3] = {x, y, z};
    const long long st[3] = {1, (long long)g.nx, (long long)g.nx * g.ny};
    const long long l = x + st[1] * y + st[2] * z;
    const float v = __ldg(img + l);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        out[d] = 0.0f;
        if (!axis_probe_inside(g, x, y, z, d, -1.0, nn[d]) ||
            !axis_probe_inside(g, x, y, z, d, +1.0, nn[d]))
            continue;
        const int p = pos[d];
        const float v2 = p < nn[d] - 1 ? fmaf(__ldg(img + l + st[d]) - v, 0.5f, v) : v;
        const float v1 = p > 0 ? fmaf(v - __ldg(img + l - st[d]), 0.5f, __ldg(img + l - st[d])) : v;
        out[d] = (float)((double)(v2 - v1) * isp[d]);
    }
}

// Thread mapping of the gather sweeps (warp, compose): a block of 256 threads is a 32 x 8 tile of
// (x, y) columns and each thread marches along z through `zchunk` slices, so the trilinear
// gathers of neighbouring columns and consecutive slices meet in L1 (the inversion step uses the
// same columns, 2 slices a tile, fw_invert.cu).
inline dim3 column_grid(int nx, int ny, int nz, int num_sms, int* zchunk) {
    dim3 g((unsigned int)((nx + 31) / 32), (unsigned int)((ny + 7) / 8), 1);
    const long long tiles = (long long)g.x * g.y;
    // about 16 blocks an SM: thin z chunks balance the SMs (measured on the 193 x 229 x 193
    // finest level: 12 chunks against 5 made compose 17 % and warp 10 % faster)
    const long long want = (16LL * num_sms + tiles - 1) / tiles;
    *zchunk = (int)((nz + (want > 1 ? want : 1) - 1) / (want > 1 ? want : 1));
    if (*zchunk < 1) *zchunk = 1;
    g.z = (unsigned int)((nz + *zchunk - 1) / *zchunk);
    return g;
}

// The thread's column of tile (bx, by, bz): x, y and the slices [z0, z1).
__device__ __forceinline__ bool column_of_tile(int nx, int ny, int nz, int zchunk, int bx, int by,
                                               int bz, int& x, int& y, int& z0, int& z1) {
    x = bx * 32 + (threadIdx.x & 31);
    y = by * 8 + (threadIdx.x >> 5);
    z0 = bz * zchunk;
    z1 = min(z0 + zchunk, nz);
    return x < nx && y < ny && z0 < z1;
}

__device__ __forceinline__ bool column_of(int nx, int ny, int nz, int zchunk, int& x, int& y,
                                          int& z0, int& z1) {
    return column_of_tile(nx, ny, nz, zchunk, blockIdx.x, blockIdx.y, blockIdx.z, x, y, z0, z1);
}

// ---- batched launches: many subjects of one level grid in one launch ---------------------
//
// The subjects of a batch share the template's level grid, so every per-subject buffer of a kind
// is one allocation with a fixed stride per subject. A batched kernel walks a work list: item w
// is tile (w mod tiles) of subject active[w / tiles]; blocks stride over the items
// (persistently: a grid of a few blocks per SM). The active list and its length live on the
// device and change between iterations (a subject that converged or failed drops out), so a
// captured graph's launches stay valid while the ragged list shrinks.
struct BatchList {
    const int* active;  // subject indices, in slot order
    const int* count;   // number of active subjects
    int tiles;          // work items per subject
};

// Tile t of a (gx, gy, *) grid as block coordinates (the single-subject kernels' blockIdx order,
// so a tile's partial sums land at the same index in both).
__device__ __forceinline__ void tile_coords(int t, int gx, int gy, int& bx, int& by, int& bz) {
    bx = t % gx;
    const int r = t / gx;
    by = r % gy;
    bz = r / gy;
}

// 32-bit division: grids hold fewer than 2^31 voxels.
__device__ __forceinline__ void voxel_ijk(long long l, int nx, int ny, int& i, int& j, int& k) {
    const unsigned int u = (unsigned int)l;
    const unsigned int q = u / (unsigned int)nx;
    i = (int)(u - q * (unsigned int)nx);
    const unsigned int kk = q / (unsigned int)ny;
    k = (int)kk;
    j = (int)(q - kk * (unsigned int)ny);
}

// non-negative float max via integer compare; NaN (canonical, positive) wins.
__device__ __forceinline__ float nan_canon(float v) {
    return isnan(v) ? __int_as_float(0x7fffffff) : v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float w = __shfl_xor_sync(0xffffffffu, v, o);
        v = __int_as_float(max(__float_as_int(v), __float_as_int(w)));
    }
    return v;
}

// The last block's fixed-order sum of `count` partials values[k * stride] (k = 0 .. count - 1),
// shared by every thread of the block (all must call it): thread t adds k = t, t + blockDim.x, ...
// in that order with four loads in flight, the warps add by shuffles and thread 0 adds the warps in
// order, so the result (valid in thread 0) does not depend on scheduling. `red` is shared scratch
// of at least blockDim.x / 32 doubles, free on entry.
__device__ __forceinline__ double block_sum_fixed(const double* values, unsigned int count,
                                                  unsigned int stride, double* red) {
    const unsigned int B = blockDim.x;
    double s = 0.0;
    unsigned int k = threadIdx.x;
    for (; k + 3 * B < count; k += 4 * B) {
        const double a0 = __ldcg(values + (size_t)k * stride);
        const double a1 = __ldcg(values + (size_t)(k + B) * stride);
        const double a2 = __ldcg(values + (size_t)(k + 2 * B) * stride);
        const double a3 = __ldcg(values + (size_t)(k + 3 * B) * stride);
        s += a0;
        s += a1;
        s += a2;
        s += a3;
    }
    for (; k < count; k += B) s += __ldcg(values + (size_t)k * stride);
    s = warp_sum_d(s);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (unsigned int w = 0; w < (B >> 5); ++w) t += red[w];
    __syncthreads();  // red is free again for the caller
    return t;
}

// The largest of `count` non-negative float64 partials values[k * stride] with NaN winning,
// shared by every thread of the block; valid in thread 0.
__device__ __forceinline__ double block_max_nan(const double* values, unsigned int count,
                                                unsigned int stride, double* red) {
    double m = 0.0;
    for (unsigned int k = threadIdx.x; k < count; k += blockDim.x) {
        const double v = __ldcg(values + (size_t)k * stride);
        m = (v > m || v != v) ? v : m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, m, o);
        m = (t > m || t != t) ? t : m;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (unsigned int w = 0; w < (blockDim.x >> 5); ++w) r = (red[w] > r || red[w] != red[w]) ? red[w] : r;
    __syncthreads();
    return r;
}

// ---- internal kernels launched by the SyN driver -------------------------------------------

// Device loop state of one inversion (fw_invert.cu).
struct InvState {
    double mean;         // MeanErrorNorm of the last measurement
    double max;          // MaxErrorNorm of the last measurement
    int executed;        // bodies executed
    int k;               // index of the next body
    int go;              // whether body k runs
    int max_iterations;
    double mean_tol, max_tol;
    int enforce;
    unsigned int lb;      // float bits: a lower bound on the running body's max error
    unsigned int ndefer;  // tiles whose update the running body left to the fix kernel
    float eps, limit;     // the last body's step and clamp (eps * max error)
    int pad;
};

// The inversion loop (fw_invert.cu). `res` (a field on the inverse's grid) keeps the residual
// of the last measurement for the body that follows.
int enqueue_inversion_prefix(fw_ctx* ctx, const fw_field* field, fw_field* inverse,
                             fw_field* res, const fw_invert_params& prm, InvState* st,
                             cudaGraphConditionalHandle handle, int use_handle);
int enqueue_inversion_body(fw_ctx* ctx, const fw_field* field, fw_field* inverse, fw_field* res,
                           InvState* st, cudaGraphConditionalHandle handle, int use_handle);
// Graph mode: scratch for an inversion's bodies without the init kernel, and the inits of up to
// kMaxInitHandles inversions (their states and WHILE conditions) in one kernel that also clears
// zero[0..nzero).
constexpr int kMaxInitHandles = 4;
int inversion_scratch(fw_ctx* ctx, const fw_field* field);
int enqueue_inversion_inits(fw_ctx* ctx, InvState* st, int count, const fw_invert_params& prm,
                            const cudaGraphConditionalHandle* handles, unsigned int* zero,
                            int nzero);
// One kernel of a body (0 bound, 1 step, 2 fix), for kernel timing.
int enqueue_inversion_kernel(fw_ctx* ctx, const fw_field* field, fw_field* inverse, fw_field* res,
                             InvState* st, int which);
long long inv_step_tiles(const HostGrid& g);
// Warp parts of the step's tiles on grid g (the capacity of a deferred list).
long long inv_step_parts(const HostGrid& g);
// Scratch doubles an inversion on grid g needs (block partials and the deferred-tile list).
size_t inv_scratch_doubles(const HostGrid& g);
long long inv_bound_voxels(const HostGrid& g);
// Adds a WHILE node on `handle` at the capture position of stream `s`; `body` receives the graph
// the loop runs (fw_syn.cu).
int add_while_node(cudaStream_t s, cudaGraphConditionalHandle handle, cudaGraph_t* body);

// Batched Gaussian smoothing of update fields (fw_smooth.cu; the same taps on the three axes,
// radius <= 12): in / out / tmp + b * stride, the max |u/sp| of subject b into
// max_bits[b * max_stride]; `blocks_xy` / `blocks_z` persistent blocks for the two passes.
int launch_smooth_batch(fw_ctx* ctx, const HostGrid& g, long long ps, double variance,
                        const int* active, const int* count, int blocks_xy, int blocks_z,
                        const float* in, float* out, float* tmp, long long stride,
                        unsigned int* max_bits, int max_stride);

// The batched inversion body (fw_invert.cu): its three kernels' work lists and persistent grids.
// Items per subject: the bound's lattice blocks, the step's blocks of `zchunk` step tiles (as the
// single step plans them, inv_step_zchunk), the fix's virtual blocks over the deferred list.
struct InvBatchBody {
    int zchunk;
    BatchList bound, step, fix;
    int bound_blocks, step_blocks, fix_blocks;
};
int inv_step_zchunk(const int64_t n[3], int num_sms);
int inv_step_blocks(const HostGrid& g, int zchunk);
int inv_bound_vblocks(const HostGrid& g);
int launch_inv_init_batch(fw_ctx* ctx, const BatchList& L, InvState* st, int st_stride,
                          const fw_invert_params& prm);
// which: -1 the whole body (bound, step, fix), else one kernel (0 bound, 1 step, 2 fix)
int launch_inv_body_batch(fw_ctx* ctx, const HostGrid& g, long long ps, const InvBatchBody& w,
                          const float* f, float* psi, float* res, long long stride,
                          double* partials, long long part_stride, unsigned int* counter,
                          InvState* st, int st_stride, unsigned int* defer,
                          long long defer_stride, int which);
// The kernel that sets the inner loop's condition (any active subject runs another body).
int launch_inv_any(fw_ctx* ctx, const InvState* st, int st_stride, const BatchList& L,
                   cudaGraphConditionalHandle handle);
int read_back(fw_ctx* ctx, const double* d, int k, double* out);
}  // namespace fw

// Device scratch of one dense Mattes MI pair (fw_mi.cu).
struct fw_dense_mi;

namespace fw {

// The dense Mattes MI pair (Backend::mi_value_derivative_pair[_masked]) as a stream-ordered
// sequence of kernels without host read-back (capturable in a graph): the two derivative fields,
// and at `publish` on the device [value (fixed, moving), |d_fixed|^2, |d_moving|^2, 0,
// value (moving, fixed), status] (status as dense_mi_status reads it).
int dense_mi_create(fw_ctx* ctx, int bins, long long n, fw_dense_mi** out);
void dense_mi_free(fw_dense_mi* d);
int enqueue_dense_mi_pair(fw_ctx* ctx, const fw_image* f, const fw_image* m, const fw_image* fm,
                          const fw_image* mm, fw_field* d_fixed, fw_field* d_moving,
                          fw_dense_mi* sc, double* publish);
// The error of a published status (0: none); `masked`: the pair had a mask.
int dense_mi_status(int status, bool masked);

// Stream-ordered host copies without a wait (the host buffer must stay valid, and for a
// download unread, until the caller synchronises): a field as AoS float32 (converted on the
// device) and an image from float32 host data.
int enqueue_field_download_f32(fw_ctx* ctx, const fw_field* field, float* host);
int enqueue_image_upload_f32(fw_ctx* ctx, const HostGrid& g, const float* host, fw_image** out);

// transform/param.rs:421-446: outer(optimised(p)) as one affine map y = M p + off (fw_mi.cu).
void linear_transform_map(const fw_linear_transform* t, double M[9], double off[3]);
// The context a device MI level evaluates on (fw_mi.cu).
const fw_ctx* mi_level_context(const fw_mi_level* level);
// A device MI level over sample records already on the device (fw_mi.cu): float32 offsets of
// the points from `center` in xyz, the fixed bin's bits in w. The level takes the moving image
// when own_moving and the records when own_rec (freed with the level, or here on failure).
int mi_level_create(fw_ctx* ctx, fw_image* moving, bool own_moving, float4* d_rec, bool own_rec,
                    int64_t n, const double center[3], const fw_mi_binning* binning,
                    fw_mi_level** out);

// A linear-stage level's prepared Mattes MI samples on the device (fw_samples.cu).
struct LevelSamples {
    float4* d_rec = nullptr;  // n records: float32 offsets from `center` in xyz, the fixed bin in w
    int64_t n = 0;
    double center[3] = {0.0, 0.0, 0.0};
    fw_mi_binning binning{};
    int64_t candidates = 0;   // sample points inside the fixed mask (every point without one)
    bool skip = false;        // Mattes MI is undefined on the level's samples: `why`
    std::string why;
};
// The regular sample set of level grid `lg` from `seed` (only the points inside `mask`, when
// given, an image on its own grid), the fixed range at their nearest voxels of `fixed`, the
// finite range of the whole `moving` image, the binning, and the records of the points whose
// trilinear fixed value exists (linear.rs:251-280, 474-492, 940-945; sampling.rs:181-238).
// Generator integers of levels generated ahead on host threads (one job per level).
struct DrawPlan {
    struct Job {
        uint32_t seed;
        int64_t picks;
        std::future<std::vector<uint32_t>> draws;
    };
    std::vector<Job> jobs;
};
// Starts generating on a host thread the draws of level grid `lg` at `percentage` from `seed`,
// unless the context holds them already.
void plan_draws(fw_ctx* ctx, DrawPlan& plan, const HostGrid& lg, float percentage, uint32_t seed);
// Returns the context's device copies of the draws to its buffer cache.
void drop_draws(fw_ctx* ctx);
int prepare_level_samples(fw_ctx* ctx, const HostGrid& lg, const fw_image* fixed,
                          const fw_image* moving, const fw_image* mask, float percentage,
                          uint32_t seed, int bins, LevelSamples& out, DrawPlan* plan = nullptr);
void free_level_samples(fw_ctx* ctx, LevelSamples& s);
// init.rs:50-74 (centre_of_gravity) over the image's float32 values, summed in float64.
int centre_of_mass(fw_ctx* ctx, const fw_image* img, double out[3]);
// Whether any voxel of the image is not zero.
int mask_has_inside(fw_ctx* ctx, const fw_image* mask, bool* any);

// The SyN recipe's validation (fw_syn.cu): 0 or FW_ERR_INVALID with the reference's message.
int syn_recipe_check(const fw_syn_recipe* r);

// The batching form (fw_batch.cu): fw_batch_syn_run after the argument checks.
int batch_syn_run(fw_ctx* ctx, const fw_syn_recipe* r, const fw_image* const* fixed, int nsub,
                  const fw_batch_subject* subj, fw_field** warps, fw_field** inverses,
                  fw_syn_iteration* records, int64_t cap, int64_t* counts, int32_t* statuses,
                  fw_batch_report* report);

// The SyN stage on device images (fw_syn.cu); masks may be null; prior / prior_inverse are the
// earlier SyN stages' collapsed fields (both null for a first stage).
int syn_run_device(fw_ctx* ctx, const fw_syn_recipe* r, const fw_image* const* fixed,
                   const fw_image* const* moving, const fw_image* fixed_mask,
                   const fw_image* moving_mask, const fw_affine* initial, const fw_field* prior,
                   const fw_field* prior_inverse, fw_field** warp, fw_field** inverse_warp,
                   fw_syn_iteration* records, int64_t cap, int64_t* count);

// d_result: [value, sum |d_fixed|^2, sum |d_moving|^2] and, with `valid` (the masked metric:
// voxels where it is not zero), the number of valid voxels at d_result[3].
int launch_cc_pair_impl(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving, int radius,
                        fw_field* d_fixed, fw_field* d_moving, double* d_result, int want_norms,
                        const fw_image* valid = nullptr);

// Gaussian taps of ITK's GaussianOperator (field_ops.rs:478-506), f64.
std::vector<double> gaussian_taps(double variance, double max_error, int64_t max_width);

// Reduction slots in ctx->d_scratch (doubles).
enum Slot : int {
    SLOT_MAX_A = 0,      // float bits of max |u/sp| (field a), as uint in a double slot
    SLOT_MAX_B = 1,
    SLOT_CC_VALUE = 2,   // -mean(localCC)
    SLOT_NORM_A = 3,     // sum u.u of derivative a
    SLOT_NORM_B = 4,
    SLOT_CC_VALID = 5,   // valid voxels of the masked CC
    SLOT_INV = 8,        // inversion state (8 doubles)
    SLOT_MI = 32,        // MI scalars
    SLOT_PARTIALS = 128, // block partials follow
};

int launch_warp(fw_ctx* ctx, const fw_image* src, const fw_field* field, const fw_field* pre,
                const fw_affine* affine, float* out, bool mask, const float* product);

// ---- batched kernels (fw_core.cu, fw_cc.cu, fw_smooth.cu, fw_invert.cu) ---------------------
// Every one runs the single-subject kernel's tile body over a BatchList with `blocks` blocks;
// per-subject buffers are base + b * stride.

// The warp arguments (an opaque device struct of warp_args_size() bytes) of a source on
// `src_grid` through a field on `field_grid` and an optional affine.
size_t warp_args_size();
void fill_warp_args(const HostGrid& src_grid, const HostGrid& field_grid, long long fps,
                    const fw_affine* affine, void* out);
int launch_warp_batch(fw_ctx* ctx, const void* d_args, const float* const* d_srcs,
                      int per_subject, const HostGrid& g, int zchunk, const BatchList& L,
                      int blocks, const float* u, long long u_stride, float* out,
                      long long out_stride);
int launch_compose_batch(fw_ctx* ctx, const HostGrid& g, long long ps, int zchunk,
                         const BatchList& L, int blocks, const float* u, float* field,
                         long long stride, const unsigned int* max_bits, int max_stride,
                         double step);
// The CC pair of a batch (unmasked): tiles per subject for z chunks of `zchunk` slices, resident
// blocks per SM, and the launch (partials: 3 doubles per tile and subject).
int cc_batch_tiles(const HostGrid& g, int zchunk);
int cc_batch_blocks_per_sm(int radius);
int launch_cc_pair_batch(fw_ctx* ctx, const HostGrid& g, long long ps, int radius, int zchunk,
                         const BatchList& L, int blocks, const float* fimg, const float* mimg,
                         long long img_stride, float* d_fixed, float* d_moving,
                         long long field_stride, double* partials, long long part_stride,
                         unsigned int* counter, double* result, int result_stride,
                         int want_norms);
int launch_cc_pair(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving, int radius,
                   fw_field* d_fixed, fw_field* d_moving, double* d_value, double* d_norms);
// Gaussian smoothing of `in` into `out` (out may be in) with the max |u/sp| of the result fused
// into d_max_bits (may be null); `tmp`, a third field on the grid, holds the xy pass (null: the
// general single-kernel path, out != in).
int launch_smooth(fw_ctx* ctx, const fw_field* in, fw_field* out, double variance,
                  unsigned int* d_max_bits, fw_field* tmp);
int launch_max_norm(fw_ctx* ctx, const fw_field* f, unsigned int* d_max_bits);
// out = a * b voxelwise (three images on one grid; out may be a or b).
int launch_image_product(fw_ctx* ctx, const fw_image* a, const fw_image* b, fw_image* out);
// out = warping + step/max * disp(x + warping) (step 1 without max bits).
int launch_compose(fw_ctx* ctx, const fw_field* disp, const fw_field* warping, fw_field* out,
                   const unsigned int* d_scale_max_bits, double step);
int launch_scale_by_max(fw_ctx* ctx, fw_field* f, const unsigned int* d_max_bits, double step);
int invert_field(fw_ctx* ctx, const fw_field* field, fw_field* inverse,
                 const fw_invert_params& prm, fw_invert_stats* stats);
int launch_resample(fw_ctx* ctx, const fw_field* f, fw_field* out);
int launch_smooth_recursive(fw_ctx* ctx, const fw_image* img, const double sigma_mm[3],
                            fw_image* out);
int reduce_l2(fw_ctx* ctx, const fw_field* f, double* d_out);

}  // namespace fw
