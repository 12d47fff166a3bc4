// fw_core.cu -- context, buffers, grids and the gather/elementwise kernels of the engine:
// warp (backend.rs:82-105), compose (backend.rs:275), resample (backend.rs:305), scale and axpy
// (backend.rs:268-271), max and L2 norms (backend.rs:252-265).
#include <cuda_runtime.h>

#include <cstdlib>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>

#include "fw_internal.cuh"

#include <chrono>
#include <thread>

namespace fw {

// ---- errors ---------------------------------------------------------------------------------

static thread_local std::string g_error;

void set_error(const std::string& msg) { g_error = msg; }

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    g_error = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
              ") in " + what;
    return e == cudaErrorMemoryAllocation ? FW_ERR_MEMORY : FW_ERR_CUDA;
}

// ---- grid math (grid.rs:45-161; linalg.rs:53-70) --------------------------------------------

bool mat3_inverse(const double m[9], double out[9]) {
    double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                 m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (det == 0.0 || !std::isfinite(det)) return false;
    double id = 1.0 / det;
    out[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    out[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    out[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    out[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    out[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    out[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    out[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    out[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    out[8] = (m[0] * m[4] - m[1] * m[3]) * id;
    return true;
}

void mat3_mul(const double a[9], const double b[9], double out[9]) {
    double t[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            t[r * 3 + c] = a[r * 3] * b[c] + a[r * 3 + 1] * b[3 + c] + a[r * 3 + 2] * b[6 + c];
    std::memcpy(out, t, sizeof(t));
}

void mat3_vec(const double m[9], const double v[3], double out[3]) {
    double t[3];
    for (int r = 0; r < 3; ++r) t[r] = m[r * 3] * v[0] + m[r * 3 + 1] * v[1] + m[r * 3 + 2] * v[2];
    out[0] = t[0];
    out[1] = t[1];
    out[2] = t[2];
}

bool HostGrid::same(const HostGrid& o) const {
    for (int a = 0; a < 3; ++a)
        if (n[a] != o.n[a] || sp[a] != o.sp[a] || org[a] != o.org[a]) return false;
    for (int a = 0; a < 9; ++a)
        if (dir[a] != o.dir[a]) return false;
    return true;
}

int make_grid(const fw_grid* g, HostGrid& out) {
    FW_CHECK(g != nullptr, "null grid");
    for (int a = 0; a < 3; ++a) {
        FW_CHECK(g->size[a] > 0, "zero size");
        FW_CHECK(g->size[a] < (1 << 20), "grid size too large");
        FW_CHECK(std::isfinite(g->spacing[a]) && g->spacing[a] > 0.0,
                 "spacing must be positive and finite");
        FW_CHECK(std::isfinite(g->origin[a]), "origin and direction must be finite");
        out.n[a] = g->size[a];
        out.sp[a] = g->spacing[a];
        out.org[a] = g->origin[a];
    }
    // voxel offsets inside a plane are 32-bit in the kernels
    FW_CHECK(out.n[0] * out.n[1] * out.n[2] < (int64_t(1) << 31),
             "grid too large: 2^31 voxels or more");
    for (int k = 0; k < 9; ++k) {
        FW_CHECK(std::isfinite(g->direction[k]), "origin and direction must be finite");
        out.dir[k] = g->direction[k];
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) out.ds[r * 3 + c] = out.dir[r * 3 + c] * out.sp[c];
    FW_CHECK(mat3_inverse(out.ds, out.inv), "singular direction matrix");
    return 0;
}

fw_grid to_c(const HostGrid& g) {
    fw_grid o;
    for (int a = 0; a < 3; ++a) {
        o.size[a] = g.n[a];
        o.spacing[a] = g.sp[a];
        o.origin[a] = g.org[a];
    }
    std::memcpy(o.direction, g.dir, sizeof(o.direction));
    return o;
}

DevGrid dev_grid(const HostGrid& g) {
    DevGrid d;
    d.nx = (int)g.n[0];
    d.ny = (int)g.n[1];
    d.nz = (int)g.n[2];
    d.n = g.count();
    for (int a = 0; a < 3; ++a) {
        d.org[a] = g.org[a];
        d.sp[a] = g.sp[a];
    }
    std::memcpy(d.ds, g.ds, sizeof(d.ds));
    std::memcpy(d.inv, g.inv, sizeof(d.inv));
    std::memcpy(d.dir, g.dir, sizeof(d.dir));
    return d;
}

// ---- buffers --------------------------------------------------------------------------------

// Sizes are rounded up to 4 KB so that buffers of nearby sizes share the cache.
static size_t cache_size(size_t bytes) { return (std::max<size_t>(bytes, 256) + 4095) & ~(size_t)4095; }

int dev_alloc(fw_ctx* ctx, size_t bytes, void** out) {
    *out = nullptr;
    const size_t sz = cache_size(bytes);
    {
        std::lock_guard<std::mutex> lock(ctx->cache_mu);
        auto it = ctx->cache.find(sz);
        if (it != ctx->cache.end()) {
            *out = it->second->p;
            ctx->cache_lru.erase(it->second);
            ctx->cache.erase(it);
            ctx->cached_bytes -= sz;
        } else if (!ctx->capturing) {
            // Requests of many grid sizes (a served stream) would otherwise leave a buffer of
            // every size they used in the cache. On a miss that would take the context past
            // twice its largest working set (at least 1 GB), buffers idle in the cache for over a
            // second go back to the pool, oldest first, which reuses their memory for any size;
            // buffers freed more recently (the same shapes about to repeat) stay. Twice: a run
            // whose levels have working sets of different sizes keeps them all for its next run
            // (a pool that gave the coarse levels' memory to the finest level would have to grow
            // for the coarse levels again). Not during a capture, where a free would become a
            // graph node.
            const uint64_t cap =
                std::max<uint64_t>(2 * ctx->stats.peak_device_bytes, (uint64_t)1 << 30);
            const auto now = std::chrono::steady_clock::now();
            while (!ctx->cache_lru.empty() &&
                   ctx->live_bytes.load() + ctx->cached_bytes + sz > cap) {
                const auto oldest = ctx->cache_lru.begin();
                if (now - oldest->freed < std::chrono::seconds(1)) break;
                auto range = ctx->cache.equal_range(oldest->size);
                for (auto m = range.first; m != range.second; ++m)
                    if (m->second == oldest) {
                        ctx->cache.erase(m);
                        break;
                    }
                cudaFreeAsync(oldest->p, ctx->stream);
                ctx->cached_bytes -= oldest->size;
                ctx->cache_lru.erase(oldest);
            }
        }
    }
    if (!*out) {
        cudaError_t e = cudaMallocFromPoolAsync(out, sz, ctx->pool, ctx->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *out = nullptr;
            return fail(FW_ERR_MEMORY, std::string("device allocation of ") + std::to_string(bytes) +
                                           " bytes failed: " + cudaGetErrorString(e));
        }
    }
    uint64_t live = ctx->live_bytes.fetch_add(sz) + sz;
    ctx->stats.live_device_bytes = live;
    if (live > ctx->stats.peak_device_bytes) ctx->stats.peak_device_bytes = live;
    return 0;
}

void dev_free(fw_ctx* ctx, void* p, size_t bytes) {
    if (!p) return;
    const size_t sz = cache_size(bytes);
    {
        std::lock_guard<std::mutex> lock(ctx->cache_mu);
        ctx->cache_lru.push_back(fw_ctx::CachedBuffer{sz, p, std::chrono::steady_clock::now()});
        ctx->cache.emplace(sz, std::prev(ctx->cache_lru.end()));
        ctx->cached_bytes += sz;
    }
    ctx->live_bytes.fetch_sub(sz);
    ctx->stats.live_device_bytes = ctx->live_bytes.load();
}

// Returns the cached buffers to the pool and the pool's unused memory to the device.
int trim_cache(fw_ctx* ctx) {
    drop_draws(ctx);
    std::list<fw_ctx::CachedBuffer> drop;
    {
        std::lock_guard<std::mutex> lock(ctx->cache_mu);
        drop.swap(ctx->cache_lru);
        ctx->cache.clear();
        ctx->cached_bytes = 0;
    }
    for (auto& c : drop) cudaFreeAsync(c.p, ctx->stream);
    FW_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->pool) FW_CUDA(cudaMemPoolTrimTo(ctx->pool, 0));
    return 0;
}

int new_image(fw_ctx* ctx, const HostGrid& g, fw_image** out) {
    fw_image* im = new fw_image{ctx, g, nullptr, (size_t)g.count() * sizeof(float)};
    int rc = dev_alloc(ctx, im->bytes, (void**)&im->d);
    if (rc) {
        delete im;
        return rc;
    }
    *out = im;
    return 0;
}

int new_field(fw_ctx* ctx, const HostGrid& g, fw_field** out) {
    int64_t ps = plane_stride(g.count());
    fw_field* f = new fw_field{ctx, g, nullptr, ps, (size_t)(3 * ps) * sizeof(float)};
    int rc = dev_alloc(ctx, f->bytes, (void**)&f->d);
    if (rc) {
        delete f;
        return rc;
    }
    *out = f;
    return 0;
}

// Waits for the context's stream on a blocking-sync event: the waiting thread sleeps instead of
// spinning, so the slots of a server do not take host cores from one another while they wait.
int sync(fw_ctx* ctx) {
    ctx->stats.host_syncs++;
    FW_CUDA(cudaEventRecord(ctx->done, ctx->stream));
    // A short wait is polled: a blocking wait sleeps until the device's interrupt wakes the
    // thread, which adds tens to hundreds of microseconds to every small read-back (the linear
    // optimiser makes thousands). The thread yields between queries, so that polling threads
    // of other contexts (the server's slots) leave the driver to the launching ones. A wait
    // longer than a millisecond then blocks and leaves the core free.
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t e = cudaEventQuery(ctx->done);
        if (e == cudaSuccess) return 0;
        if (e != cudaErrorNotReady) return cuda_fail(e, "cudaEventQuery");
        if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(1)) break;
        std::this_thread::yield();
    }
    FW_CUDA(cudaEventSynchronize(ctx->done));
    return 0;
}

int host_stage(fw_ctx* ctx, size_t bytes, void** out) {
    if (bytes > ctx->h_stage_bytes) {
        if (ctx->h_stage) {
            FW_TRY(sync(ctx));
            cudaFreeHost(ctx->h_stage);
            ctx->h_stage = nullptr;
            ctx->h_stage_bytes = 0;
        }
        const size_t want = std::max<size_t>(bytes, (size_t)1 << 20);
        if (cudaMallocHost(&ctx->h_stage, want) != cudaSuccess) {
            cudaGetLastError();
            ctx->h_stage = nullptr;
            return fail(FW_ERR_MEMORY, "pinned staging allocation failed");
        }
        ctx->h_stage_bytes = want;
    }
    *out = ctx->h_stage;
    return 0;
}

bool pdl_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("FASTWARP_PDL");
        return !(v && v[0] == '0');
    }();
    return on;
}

int check_launch(fw_ctx* ctx, const char* what) {
    ctx->stats.kernel_launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what);
    return 0;
}

int ensure_scratch(fw_ctx* ctx, size_t doubles) {
    if (doubles <= ctx->scratch_doubles) return 0;
    if (ctx->capturing) return fail(FW_ERR_INVALID, "scratch too small for a graph capture");
    if (ctx->d_scratch) {
        FW_CUDA(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->d_scratch);
        ctx->d_scratch = nullptr;
    }
    size_t n = std::max<size_t>(doubles, 1 << 16);
    FW_CUDA(cudaMalloc(&ctx->d_scratch, n * sizeof(double)));
    FW_CUDA(cudaMemset(ctx->d_scratch, 0, n * sizeof(double)));
    ctx->scratch_doubles = n;
    return 0;
}

// ---- kernels --------------------------------------------------------------------------------

struct WarpArgs {
    DevGrid g;        // output grid (the field's)
    DevGrid s;        // source grid
    DevGrid p;        // grid of `pre`
    double q[9];      // source index from output index (no `pre`)
    double r[9];      // source index from displacement (no `pre`)
    double q0[3];
    double am[9];     // affine matrix (identity when absent)
    double ao[3];
    int has_pre;
    int mask;
    long long fps;    // plane stride of the field
    long long pps;    // plane stride of `pre`
};

// cpu/mod.rs:60-132: out(x) = src(affine(q + pre(q))), q = x + u(x); linear (ITK scalar rule,
// zero outside) or nearest voxel of a mask (rounding half up).
__global__ void __launch_bounds__(256) k_warp(WarpArgs a, const float* __restrict__ u,
                                              const float* __restrict__ pre,
                                              const float* __restrict__ src,
                                              const float* product, float* out) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= a.g.n) return;
    int i, j, k;
    voxel_ijk(l, a.g.nx, a.g.ny, i, j, k);
    double ux = u[l], uy = u[l + a.fps], uz = u[l + 2 * a.fps];
    double c[3];
    if (!a.has_pre) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
            c[r] = a.q[r * 3] * i + a.q[r * 3 + 1] * j + a.q[r * 3 + 2] * k + a.q0[r] +
                   (a.r[r * 3] * ux + a.r[r * 3 + 1] * uy + a.r[r * 3 + 2] * uz);
    } else {
        double p[3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
            p[r] = a.g.org[r] + (a.g.ds[r * 3] * i + a.g.ds[r * 3 + 1] * j + a.g.ds[r * 3 + 2] * k);
        p[0] += ux;
        p[1] += uy;
        p[2] += uz;
        double d0 = p[0] - a.p.org[0], d1 = p[1] - a.p.org[1], d2 = p[2] - a.p.org[2];
        double pc[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) pc[r] = a.p.inv[r * 3] * d0 + a.p.inv[r * 3 + 1] * d1 + a.p.inv[r * 3 + 2] * d2;
        if (inside_index(pc[0], pc[1], pc[2], a.p.nx, a.p.ny, a.p.nz)) {
            float d[3];
            vec_at_index(pre, a.pps, a.p.nx, a.p.ny, a.p.nz, pc[0], pc[1], pc[2], d);
            p[0] += d[0];
            p[1] += d[1];
            p[2] += d[2];
        }
        double t[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) t[r] = a.am[r * 3] * p[0] + a.am[r * 3 + 1] * p[1] + a.am[r * 3 + 2] * p[2] + a.ao[r];
        double e0 = t[0] - a.s.org[0], e1 = t[1] - a.s.org[1], e2 = t[2] - a.s.org[2];
#pragma unroll
        for (int r = 0; r < 3; ++r) c[r] = a.s.inv[r * 3] * e0 + a.s.inv[r * 3 + 1] * e1 + a.s.inv[r * 3 + 2] * e2;
    }
    float v = 0.0f;
    if (a.mask) {
        double rx = floor(c[0] + 0.5), ry = floor(c[1] + 0.5), rz = floor(c[2] + 0.5);
        if (rx >= 0.0 && rx < a.s.nx && ry >= 0.0 && ry < a.s.ny && rz >= 0.0 && rz < a.s.nz) {
            long long m = (long long)rx + (long long)a.s.nx * ((long long)ry + (long long)a.s.ny * (long long)rz);
            v = __ldg(src + m) != 0.0f ? 1.0f : 0.0f;
        }
        if (product) v *= product[l];
    } else if (inside_index(c[0], c[1], c[2], a.s.nx, a.s.ny, a.s.nz)) {
        v = lin_at_index(src, a.s.nx, a.s.ny, a.s.nz, c[0], c[1], c[2]);
    }
    out[l] = v;
}

// The plain warp (no earlier field, linear interpolation) -- the SyN loop's per-iteration warps --
// over 32 x 8 column tiles marching along z, the next slice's displacement loaded while the
// current one gathers. One column [z0, z1) of the thread.
__device__ __forceinline__ void warp_column(const WarpArgs& a, int x, int y, int z0, int z1,
                                            const float* __restrict__ u,
                                            const float* __restrict__ src,
                                            float* __restrict__ out) {
    const long long sxy = (long long)a.g.nx * a.g.ny;
    long long l = (long long)z0 * sxy + (long long)y * a.g.nx + x;
    float ux = u[l], uy = u[l + a.fps], uz = u[l + 2 * a.fps];
    const double xd = (double)x, yd = (double)y;  // converted once (the conversions are slow)
    double kd = (double)z0;
    for (int k = z0; k < z1; ++k, l += sxy, kd += 1.0) {
        float nx_ = 0.0f, ny_ = 0.0f, nz_ = 0.0f;
        if (k + 1 < z1) {
            nx_ = u[l + sxy];
            ny_ = u[l + sxy + a.fps];
            nz_ = u[l + sxy + 2 * a.fps];
        }
        double c[3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
            c[r] = a.q[r * 3] * xd + a.q[r * 3 + 1] * yd + a.q[r * 3 + 2] * kd + a.q0[r] +
                   (a.r[r * 3] * ux + a.r[r * 3 + 1] * uy + a.r[r * 3 + 2] * uz);
        float v = 0.0f;
        if (inside_index(c[0], c[1], c[2], a.s.nx, a.s.ny, a.s.nz))
            v = lin_at_index(src, a.s.nx, a.s.ny, a.s.nz, c[0], c[1], c[2]);
        out[l] = v;
        ux = nx_;
        uy = ny_;
        uz = nz_;
    }
}

__global__ void __launch_bounds__(256) k_warp_t(WarpArgs a, int zchunk,
                                                const float* __restrict__ u,
                                                const float* __restrict__ src,
                                                float* __restrict__ out) {
    pdl_wait();
    int x, y, z0, z1;
    if (!column_of(a.g.nx, a.g.ny, a.g.nz, zchunk, x, y, z0, z1)) return;
    warp_column(a, x, y, z0, z1, u, src, out);
}

// The same warp for every active subject of a batch: subject b gathers from srcs[b] through
// args[b] (per_subject) or from srcs[0] through args[0] (the shared template), with its field at
// u + b * u_stride and its output at out + b * out_stride.
__global__ void __launch_bounds__(256) k_warp_t_batch(const WarpArgs* __restrict__ args,
                                                      const float* const* __restrict__ srcs,
                                                      int per_subject, int zchunk, BatchList L,
                                                      const float* __restrict__ u,
                                                      long long u_stride,
                                                      float* __restrict__ out,
                                                      long long out_stride) {
    const int work = *L.count * L.tiles;
    const int gx = (args[0].g.nx + 31) / 32, gy = (args[0].g.ny + 7) / 8;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles];
        const int q = per_subject ? b : 0;
        const WarpArgs& a = args[q];
        int bx, by, bz, x, y, z0, z1;
        tile_coords(w % L.tiles, gx, gy, bx, by, bz);
        if (!column_of_tile(a.g.nx, a.g.ny, a.g.nz, zchunk, bx, by, bz, x, y, z0, z1)) continue;
        warp_column(a, x, y, z0, z1, u + b * u_stride, srcs[q], out + b * out_stride);
    }
}

struct FieldArgs {
    DevGrid g;
    long long ps;
};

// field_ops.rs:251-272 with the scale of syn.rs:285-298 fused: out(x) = w(x) + s * u(x + w(x)),
// s = step / max |u/sp| (step when the max is 0) or 1 without a max.
// `w` and `out` may be the same buffer (the SyN loop composes in place: a voxel reads only its
// own value of `w`), so neither is declared __restrict__. One column [z0, z1) of the thread.
__device__ __forceinline__ void compose_column(const FieldArgs& a, int i, int j, int z0, int z1,
                                               const float* __restrict__ u, const float* w,
                                               float* out,
                                               const unsigned int* __restrict__ max_bits,
                                               double step) {
    float s = 1.0f;
    if (max_bits) {
        float mx = __uint_as_float(*max_bits);
        s = mx > 0.0f ? (float)(step / (double)mx) : (float)step;
    }
    const long long sxy = (long long)a.g.nx * a.g.ny;
    long long l = (long long)z0 * sxy + (long long)j * a.g.nx + i;
    float wx = w[l], wy = w[l + a.ps], wz = w[l + 2 * a.ps];
    for (int k = z0; k < z1; ++k, l += sxy) {
        // the next slice's own field values, in flight during this slice's gather (each voxel
        // reads only its own w, so the composition may run in place)
        float qx = 0.0f, qy = 0.0f, qz = 0.0f;
        if (k + 1 < z1) {
            qx = w[l + sxy];
            qy = w[l + sxy + a.ps];
            qz = w[l + sxy + 2 * a.ps];
        }
        double c[3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
            c[r] = (r == 0 ? i : (r == 1 ? j : k)) +
                   (a.g.inv[r * 3] * wx + a.g.inv[r * 3 + 1] * wy + a.g.inv[r * 3 + 2] * wz);
        float d[3] = {0.0f, 0.0f, 0.0f};
        if (inside_index(c[0], c[1], c[2], a.g.nx, a.g.ny, a.g.nz))
            vec_at_index(u, a.ps, a.g.nx, a.g.ny, a.g.nz, c[0], c[1], c[2], d);
        out[l] = fmaf(s, d[0], wx);
        out[l + a.ps] = fmaf(s, d[1], wy);
        out[l + 2 * a.ps] = fmaf(s, d[2], wz);
        wx = qx;
        wy = qy;
        wz = qz;
    }
}

__global__ void __launch_bounds__(256) k_compose(FieldArgs a, int zchunk,
                                                 const float* __restrict__ u, const float* w,
                                                 float* out,
                                                 const unsigned int* __restrict__ max_bits,
                                                 double step) {
    pdl_wait();
    int i, j, z0, z1;
    if (!column_of(a.g.nx, a.g.ny, a.g.nz, zchunk, i, j, z0, z1)) return;
    compose_column(a, i, j, z0, z1, u, w, out, max_bits, step);
}

// In place for every active subject of a batch: field + b * stride composed with the update
// u + b * stride, scaled by step / its max at max_bits[b * max_stride].
__global__ void __launch_bounds__(256) k_compose_batch(FieldArgs a, int zchunk, BatchList L,
                                                       const float* __restrict__ u, float* field,
                                                       long long stride,
                                                       const unsigned int* __restrict__ max_bits,
                                                       int max_stride, double step) {
    const int work = *L.count * L.tiles;
    const int gx = (a.g.nx + 31) / 32, gy = (a.g.ny + 7) / 8;
    for (int w = blockIdx.x; w < work; w += gridDim.x) {
        const int b = L.active[w / L.tiles];
        int bx, by, bz, i, j, z0, z1;
        tile_coords(w % L.tiles, gx, gy, bx, by, bz);
        if (!column_of_tile(a.g.nx, a.g.ny, a.g.nz, zchunk, bx, by, bz, i, j, z0, z1)) continue;
        float* f = field + b * stride;
        compose_column(a, i, j, z0, z1, u + b * stride, f, f, max_bits + b * max_stride, step);
    }
}

// field_ops.rs:580-605: onto another grid, scalar linear interpolation per component, zero
// outside the old buffer.
__global__ void __launch_bounds__(256) k_resample(DevGrid d, DevGrid s, const float* __restrict__ f,
                                                  long long fps, float* __restrict__ out,
                                                  long long ops) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= d.n) return;
    int i, j, k;
    voxel_ijk(l, d.nx, d.ny, i, j, k);
    double p[3], c[3];
    exact_point(d, i, j, k, p);
    exact_index(s, p, c);
    bool in = inside_index(c[0], c[1], c[2], s.nx, s.ny, s.nz);
#pragma unroll
    for (int q = 0; q < 3; ++q)
        out[l + q * ops] = in ? lin_at_index(f + q * fps, s.nx, s.ny, s.nz, c[0], c[1], c[2]) : 0.0f;
}

// field_ops.rs:191-203: atomic max of |u/sp| as float bits (non-negative; NaN wins).
__global__ void __launch_bounds__(256) k_max_norm(FieldArgs a, const float* __restrict__ u,
                                                  unsigned int* __restrict__ max_bits) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float v = 0.0f;
    if (l < a.g.n) {
        float x = u[l] / (float)a.g.sp[0], y = u[l + a.ps] / (float)a.g.sp[1],
              z = u[l + 2 * a.ps] / (float)a.g.sp[2];
        v = nan_canon(sqrtf(x * x + y * y + z * z));
    }
    v = warp_max_f(v);
    if ((threadIdx.x & 31) == 0 && v > 0.0f) atomicMax(max_bits, __float_as_uint(v));
}

// Fixed-order last-block reduction: every block writes `k` partials at its index; the last
// block to finish sums them in block order, so the result does not depend on scheduling.
__device__ bool is_last_block(unsigned int* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    return last;
}

// field_ops.rs:205-213: sum of u.u in f64.
__global__ void __launch_bounds__(256) k_l2(FieldArgs a, const float* __restrict__ u,
                                            double* __restrict__ partials,
                                            unsigned int* __restrict__ counter,
                                            double* __restrict__ result) {
    __shared__ double red[8];
    double acc = 0.0;
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < a.g.n;
         l += (long long)gridDim.x * blockDim.x) {
        double x = u[l], y = u[l + a.ps], z = u[l + 2 * a.ps];
        acc += x * x + y * y + z * z;
    }
    acc = warp_sum_d(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        partials[blockIdx.x] = s;
    }
    if (!is_last_block(counter)) return;
    double s = 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += __ldcg(partials + b);
    s = warp_sum_d(s);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        *result = t;
        *counter = 0;
    }
}

__global__ void k_scale(float4* __restrict__ f, long long n4, float s) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n4) return;
    float4 v = f[l];
    v.x *= s;
    v.y *= s;
    v.z *= s;
    v.w *= s;
    f[l] = v;
}

__global__ void k_scale_by_max(float4* __restrict__ f, long long n4,
                               const unsigned int* __restrict__ max_bits, double step) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n4) return;
    float mx = __uint_as_float(*max_bits);
    float s = mx > 0.0f ? (float)(step / (double)mx) : (float)step;
    float4 v = f[l];
    v.x *= s;
    v.y *= s;
    v.z *= s;
    v.w *= s;
    f[l] = v;
}

__global__ void k_axpy(float4* __restrict__ acc, const float4* __restrict__ x, long long n4,
                       float a) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n4) return;
    float4 v = acc[l], w = x[l];
    v.x = fmaf(a, w.x, v.x);
    v.y = fmaf(a, w.y, v.y);
    v.z = fmaf(a, w.z, v.z);
    v.w = fmaf(a, w.w, v.w);
    acc[l] = v;
}

// ---- launchers ------------------------------------------------------------------------------

static inline unsigned int blocks_for(long long n, int t = 256) {
    return (unsigned int)((n + t - 1) / t);
}

// The arguments of a warp of a source on `sg` through a field on `fg` (plane stride fps) and an
// optional affine, without an earlier field: the index map c = Q idx + R u + q0.
static void plain_warp_args(const HostGrid& sg, const HostGrid& fg, long long fps,
                            const fw_affine* affine, WarpArgs& a) {
    std::memset(&a, 0, sizeof(a));
    a.g = dev_grid(fg);
    a.s = dev_grid(sg);
    a.fps = fps;
    double am[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, ao[3] = {0, 0, 0};
    if (affine) {
        std::memcpy(am, affine->matrix, sizeof(am));
        std::memcpy(ao, affine->offset, sizeof(ao));
    }
    std::memcpy(a.am, am, sizeof(am));
    std::memcpy(a.ao, ao, sizeof(ao));
    // c = S^-1 (A (org + DS idx + u) + ao - s_org) = Q idx + R u + q0
    double ra[9];
    mat3_mul(sg.inv, am, ra);
    mat3_mul(ra, fg.ds, a.q);
    std::memcpy(a.r, ra, sizeof(ra));
    double ag[3];
    mat3_vec(am, fg.org, ag);
    double t[3] = {ag[0] + ao[0] - sg.org[0], ag[1] + ao[1] - sg.org[1], ag[2] + ao[2] - sg.org[2]};
    mat3_vec(sg.inv, t, a.q0);
}

size_t warp_args_size() { return sizeof(WarpArgs); }

void fill_warp_args(const HostGrid& src_grid, const HostGrid& field_grid, long long fps,
                    const fw_affine* affine, void* out) {
    plain_warp_args(src_grid, field_grid, fps, affine, *static_cast<WarpArgs*>(out));
}

int launch_warp_batch(fw_ctx* ctx, const void* d_args, const float* const* d_srcs,
                      int per_subject, const HostGrid& g, int zchunk, const BatchList& L,
                      int blocks, const float* u, long long u_stride, float* out,
                      long long out_stride) {
    (void)g;
    k_warp_t_batch<<<blocks, 256, 0, ctx->stream>>>(static_cast<const WarpArgs*>(d_args), d_srcs,
                                                   per_subject, zchunk, L, u, u_stride, out,
                                                   out_stride);
    return check_launch(ctx, "k_warp_t_batch");
}

int launch_compose_batch(fw_ctx* ctx, const HostGrid& g, long long ps, int zchunk,
                         const BatchList& L, int blocks, const float* u, float* field,
                         long long stride, const unsigned int* max_bits, int max_stride,
                         double step) {
    FieldArgs a{dev_grid(g), ps};
    k_compose_batch<<<blocks, 256, 0, ctx->stream>>>(a, zchunk, L, u, field, stride, max_bits,
                                                    max_stride, step);
    return check_launch(ctx, "k_compose_batch");
}

int launch_warp(fw_ctx* ctx, const fw_image* src, const fw_field* field, const fw_field* pre,
                const fw_affine* affine, float* out, bool mask, const float* product) {
    WarpArgs a;
    plain_warp_args(src->grid, field->grid, field->ps, affine, a);
    a.mask = mask ? 1 : 0;
    if (pre) {
        a.has_pre = 1;
        a.p = dev_grid(pre->grid);
        a.pps = pre->ps;
    }
    long long n = a.g.n;
    if (!pre && !mask) {
        int zchunk = 1;
        const dim3 grid = column_grid(a.g.nx, a.g.ny, a.g.nz, ctx->num_sms, &zchunk);
        return launch_pdl(ctx, "k_warp_t", k_warp_t, grid, dim3(256), 0, a, zchunk,
                          (const float*)field->d, (const float*)src->d, out);
    }
    k_warp<<<blocks_for(n), 256, 0, ctx->stream>>>(a, field->d, pre ? pre->d : nullptr, src->d,
                                                   product, out);
    return check_launch(ctx, "k_warp");
}

int launch_compose(fw_ctx* ctx, const fw_field* disp, const fw_field* warping, fw_field* out,
                   const unsigned int* d_scale_max_bits, double step) {
    FieldArgs a{dev_grid(warping->grid), warping->ps};
    int zchunk = 1;
    const dim3 grid = column_grid(a.g.nx, a.g.ny, a.g.nz, ctx->num_sms, &zchunk);
    return launch_pdl(ctx, "k_compose", k_compose, grid, dim3(256), 0, a, zchunk,
                      (const float*)disp->d, (const float*)warping->d, out->d, d_scale_max_bits,
                      step);
}

__global__ void k_image_product(const float* __restrict__ a, const float* __restrict__ b,
                                float* __restrict__ out, long long n) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l < n) out[l] = a[l] * b[l];
}

int launch_image_product(fw_ctx* ctx, const fw_image* a, const fw_image* b, fw_image* out) {
    long long n = out->grid.count();
    k_image_product<<<blocks_for(n), 256, 0, ctx->stream>>>(a->d, b->d, out->d, n);
    return check_launch(ctx, "k_image_product");
}

int launch_max_norm(fw_ctx* ctx, const fw_field* f, unsigned int* d_max_bits) {
    FieldArgs a{dev_grid(f->grid), f->ps};
    k_max_norm<<<blocks_for(a.g.n), 256, 0, ctx->stream>>>(a, f->d, d_max_bits);
    return check_launch(ctx, "k_max_norm");
}

int launch_scale_by_max(fw_ctx* ctx, fw_field* f, const unsigned int* d_max_bits, double step) {
    long long n4 = 3 * f->ps / 4;
    k_scale_by_max<<<blocks_for(n4), 256, 0, ctx->stream>>>((float4*)f->d, n4, d_max_bits, step);
    return check_launch(ctx, "k_scale_by_max");
}

int launch_resample(fw_ctx* ctx, const fw_field* f, fw_field* out) {
    DevGrid d = dev_grid(out->grid), s = dev_grid(f->grid);
    k_resample<<<blocks_for(d.n), 256, 0, ctx->stream>>>(d, s, f->d, f->ps, out->d, out->ps);
    return check_launch(ctx, "k_resample");
}

int reduce_l2(fw_ctx* ctx, const fw_field* f, double* d_out) {
    FieldArgs a{dev_grid(f->grid), f->ps};
    unsigned int blocks = std::min<unsigned int>(blocks_for(a.g.n), 4u * ctx->num_sms);
    FW_TRY(ensure_scratch(ctx, SLOT_PARTIALS + blocks + 16));
    k_l2<<<blocks, 256, 0, ctx->stream>>>(a, f->d, ctx->d_scratch + SLOT_PARTIALS, ctx->d_counter,
                                          d_out);
    return check_launch(ctx, "k_l2");
}

// Reads `k` doubles from device scratch into pinned memory and waits.
static int read_scalars(fw_ctx* ctx, const double* d, int k, double* out) {
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, d, sizeof(double) * k, cudaMemcpyDeviceToHost,
                            ctx->stream));
    FW_TRY(sync(ctx));
    ctx->stats.bytes_downloaded += sizeof(double) * k;
    for (int i = 0; i < k; ++i) out[i] = ctx->h_pinned[i];
    return 0;
}

int read_back(fw_ctx* ctx, const double* d, int k, double* out) { return read_scalars(ctx, d, k, out); }

}  // namespace fw

using namespace fw;

// ---- C ABI ----------------------------------------------------------------------------------

extern "C" {

const char* fw_last_error(void) { return fw::g_error.c_str(); }

const char* fw_backend_name(void) { return "cuda-sm100a-f32"; }

int fw_ctx_create(int device, fw_ctx** out) {
    FW_CHECK(out != nullptr, "null output");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(FW_ERR_CUDA, "no CUDA device is available (this engine has no CPU fallback)");
    }
    FW_CHECK(device >= 0 && device < count, "device index out of range");
    FW_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    FW_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return fail(FW_ERR_CUDA, std::string("device ") + prop.name +
                                     " is not sm_100 (this library is built for sm_100a only)");
    fw_ctx* ctx = new fw_ctx();
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&ctx->done, cudaEventBlockingSync | cudaEventDisableTiming);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(e, "cudaStreamCreate");
    }
    // a memory pool of the context's own that keeps freed blocks (the buffer pool of the wgpu
    // engine, pool.rs): every allocation and free is ordered on the context's stream, so after
    // the first registration of a shape the next ones reuse the same blocks; a pool shared with
    // other streams could not always reuse them and would grow instead
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    e = cudaMemPoolCreate(&ctx->pool, &props);
    if (e == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        fw_ctx_destroy(ctx);
        return cuda_fail(e, "cudaMemPoolCreate");
    }
    if (cudaMalloc(&ctx->d_counter, 64 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMemset(ctx->d_counter, 0, 64 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_pinned, 4096 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        fw_ctx_destroy(ctx);
        return fail(FW_ERR_MEMORY, "context scratch allocation failed");
    }
    // the cancel flag the device can read: one int of mapped pinned host memory
    void* flag = nullptr;
    void* flag_dev = nullptr;
    if (cudaHostAlloc(&flag, 64, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
        cudaHostGetDevicePointer(&flag_dev, flag, 0) != cudaSuccess) {
        cudaGetLastError();
        if (flag) cudaFreeHost(flag);
        fw_ctx_destroy(ctx);
        return fail(FW_ERR_MEMORY, "context cancel flag allocation failed");
    }
    ctx->cancel_mapped = static_cast<volatile int32_t*>(flag);
    *ctx->cancel_mapped = 0;
    ctx->cancel_mapped_dev = static_cast<const volatile int32_t*>(flag_dev);
    int rc = ensure_scratch(ctx, 1 << 16);
    if (rc) {
        fw_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return 0;
}

void fw_ctx_destroy(fw_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    drop_draws(ctx);
    if (ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        for (auto& c : ctx->cache_lru) cudaFreeAsync(c.p, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
    }
    ctx->cache.clear();
    ctx->cache_lru.clear();
    if (ctx->d_scratch) cudaFree(ctx->d_scratch);
    if (ctx->d_counter) cudaFree(ctx->d_counter);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    if (ctx->cancel_mapped) cudaFreeHost(const_cast<int32_t*>(ctx->cancel_mapped));
    if (ctx->done) cudaEventDestroy(ctx->done);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->aux) cudaStreamDestroy(ctx->aux);
    // the pool's blocks go back to the device; a buffer still outstanding keeps them until freed
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

int fw_ctx_release_idle_buffers(fw_ctx* ctx) {
    FW_CHECK(ctx, "null context");
    return trim_cache(ctx);
}

int fw_ctx_cached_bytes(const fw_ctx* ctx, uint64_t* out) {
    FW_CHECK(ctx && out, "null argument");
    std::lock_guard<std::mutex> lock(const_cast<fw_ctx*>(ctx)->cache_mu);
    *out = ctx->cached_bytes;
    return 0;
}

void* fw_ctx_stream(fw_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int fw_ctx_synchronize(fw_ctx* ctx) {
    FW_CHECK(ctx, "null context");
    return sync(ctx);
}

int fw_ctx_stats(const fw_ctx* ctx, fw_stats* out) {
    FW_CHECK(ctx && out, "null argument");
    *out = ctx->stats;
    return 0;
}

void fw_ctx_reset_stats(fw_ctx* ctx) {
    if (!ctx) return;
    uint64_t live = ctx->live_bytes.load();
    std::memset(&ctx->stats, 0, sizeof(ctx->stats));
    ctx->stats.live_device_bytes = live;
    ctx->stats.peak_device_bytes = live;
}

int fw_ctx_set_cancel_flag(fw_ctx* ctx, const volatile int32_t* flag) {
    FW_CHECK(ctx, "null context");
    ctx->cancel = flag;
    return 0;
}

int fw_ctx_request_cancel(fw_ctx* ctx, int32_t on) {
    FW_CHECK(ctx && ctx->cancel_mapped, "null context");
    *ctx->cancel_mapped = on ? 1 : 0;
    return 0;
}

int fw_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes) {
    FW_CUDA(cudaSetDevice(device));
    size_t f = 0, t = 0;
    FW_CUDA(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return 0;
}

// -- images

int fw_image_upload_f32(fw_ctx* ctx, const fw_grid* grid, const float* host, fw_image** out) {
    FW_CHECK(ctx && host && out, "null argument");
    HostGrid g;
    FW_TRY(make_grid(grid, g));
    fw_image* im;
    FW_TRY(new_image(ctx, g, &im));
    cudaError_t e = cudaMemcpyAsync(im->d, host, im->bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        fw_image_free(im);
        return cuda_fail(e, "image upload");
    }
    ctx->stats.bytes_uploaded += im->bytes;
    int rc = sync(ctx);
    if (rc) {
        fw_image_free(im);
        return rc;
    }
    *out = im;
    return 0;
}

int fw_image_upload(fw_ctx* ctx, const fw_grid* grid, const double* host, fw_image** out) {
    FW_CHECK(ctx && host && out, "null argument");
    HostGrid g;
    FW_TRY(make_grid(grid, g));
    std::vector<float> tmp((size_t)g.count());
    for (size_t i = 0; i < tmp.size(); ++i) tmp[i] = (float)host[i];
    return fw_image_upload_f32(ctx, grid, tmp.data(), out);
}

int fw_image_download(fw_ctx* ctx, const fw_image* img, float* host) {
    FW_CHECK(ctx && img && host, "null argument");
    FW_CUDA(cudaMemcpyAsync(host, img->d, img->bytes, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->stats.bytes_downloaded += img->bytes;
    return sync(ctx);
}

int fw_image_grid(const fw_image* img, fw_grid* out) {
    FW_CHECK(img && out, "null argument");
    *out = to_c(img->grid);
    return 0;
}

void* fw_image_device_ptr(fw_image* img) { return img ? img->d : nullptr; }

void fw_image_free(fw_image* img) {
    if (!img) return;
    dev_free(img->ctx, img->d, img->bytes);
    delete img;
}

// -- fields

int fw_field_zero(fw_ctx* ctx, const fw_grid* grid, fw_field** out) {
    FW_CHECK(ctx && out, "null argument");
    HostGrid g;
    FW_TRY(make_grid(grid, g));
    fw_field* f;
    FW_TRY(new_field(ctx, g, &f));
    cudaError_t e = cudaMemsetAsync(f->d, 0, f->bytes, ctx->stream);
    if (e != cudaSuccess) {
        fw_field_free(f);
        return cuda_fail(e, "field memset");
    }
    *out = f;
    return 0;
}

int fw_field_upload(fw_ctx* ctx, const fw_grid* grid, const double* aos, fw_field** out) {
    FW_CHECK(ctx && aos && out, "null argument");
    HostGrid g;
    FW_TRY(make_grid(grid, g));
    fw_field* f;
    FW_TRY(new_field(ctx, g, &f));
    int64_t n = g.count();
    std::vector<float> soa((size_t)(3 * f->ps), 0.0f);
    for (int64_t l = 0; l < n; ++l)
        for (int c = 0; c < 3; ++c) soa[c * f->ps + l] = (float)aos[3 * l + c];
    cudaError_t e = cudaMemcpyAsync(f->d, soa.data(), f->bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        fw_field_free(f);
        return cuda_fail(e, "field upload");
    }
    ctx->stats.bytes_uploaded += f->bytes;
    int rc = sync(ctx);
    if (rc) {
        fw_field_free(f);
        return rc;
    }
    *out = f;
    return 0;
}

}  // extern "C"

namespace fw {
namespace {

// SoA planes -> AoS (x, y, z per voxel) of float or double, on the device.
template <typename T>
__global__ void k_soa_to_aos(const float* __restrict__ f, long long ps, long long n,
                             T* __restrict__ out) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n) return;
    out[3 * l] = (T)f[l];
    out[3 * l + 1] = (T)f[l + ps];
    out[3 * l + 2] = (T)f[l + 2 * ps];
}

template <typename T>
int enqueue_field_aos(fw_ctx* ctx, const fw_field* field, T* host) {
    const long long n = field->grid.count();
    const size_t bytes = sizeof(T) * 3 * (size_t)n;
    void* tmp = nullptr;
    FW_TRY(dev_alloc(ctx, bytes, &tmp));
    k_soa_to_aos<T><<<blocks_for(n), 256, 0, ctx->stream>>>(field->d, field->ps, n,
                                                            static_cast<T*>(tmp));
    int rc = check_launch(ctx, "k_soa_to_aos");
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "field download");
    }
    ctx->stats.bytes_downloaded += bytes;
    dev_free(ctx, tmp, bytes);  // reused only by later work on this stream
    return rc;
}

}  // namespace

int enqueue_field_download_f32(fw_ctx* ctx, const fw_field* field, float* host) {
    return enqueue_field_aos<float>(ctx, field, host);
}

int enqueue_image_upload_f32(fw_ctx* ctx, const HostGrid& g, const float* host, fw_image** out) {
    fw_image* im;
    FW_TRY(new_image(ctx, g, &im));
    cudaError_t e = cudaMemcpyAsync(im->d, host, im->bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        fw_image_free(im);
        return cuda_fail(e, "image upload");
    }
    ctx->stats.bytes_uploaded += im->bytes;
    *out = im;
    return 0;
}

}  // namespace fw

extern "C" {

int fw_field_download(fw_ctx* ctx, const fw_field* field, double* aos) {
    FW_CHECK(ctx && field && aos, "null argument");
    FW_TRY(enqueue_field_aos<double>(ctx, field, aos));
    return sync(ctx);
}

int fw_field_download_f32(fw_ctx* ctx, const fw_field* field, float* aos) {
    FW_CHECK(ctx && field && aos, "null argument");
    FW_TRY(enqueue_field_aos<float>(ctx, field, aos));
    return sync(ctx);
}

int fw_field_grid(const fw_field* field, fw_grid* out) {
    FW_CHECK(field && out, "null argument");
    *out = to_c(field->grid);
    return 0;
}

int fw_field_copy(fw_ctx* ctx, const fw_field* field, fw_field** out) {
    FW_CHECK(ctx && field && out, "null argument");
    fw_field* f;
    FW_TRY(new_field(ctx, field->grid, &f));
    cudaError_t e = cudaMemcpyAsync(f->d, field->d, f->bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) {
        fw_field_free(f);
        return cuda_fail(e, "field copy");
    }
    *out = f;
    return sync(ctx);
}

void* fw_field_device_ptr(fw_field* field, int64_t* plane_stride) {
    if (!field) return nullptr;
    if (plane_stride) *plane_stride = field->ps;
    return field->d;
}

void fw_field_free(fw_field* field) {
    if (!field) return;
    dev_free(field->ctx, field->d, field->bytes);
    delete field;
}

// -- operations

int fw_warp_through_field(fw_ctx* ctx, const fw_image* source, const fw_field* field,
                          const fw_field* pre, const fw_affine* affine, fw_image** out) {
    FW_CHECK(ctx && source && field && out, "null argument");
    fw_image* im;
    FW_TRY(new_image(ctx, field->grid, &im));
    int rc = launch_warp(ctx, source, field, pre, affine, im->d, false, nullptr);
    if (!rc) rc = sync(ctx);
    if (rc) {
        fw_image_free(im);
        return rc;
    }
    *out = im;
    return 0;
}

int fw_warp_mask_through_field(fw_ctx* ctx, const fw_image* mask, const fw_field* field,
                               const fw_field* pre, const fw_affine* affine, fw_image* product,
                               fw_image** out) {
    FW_CHECK(ctx && mask && field && out, "null argument");
    if (product && !product->grid.same(field->grid))
        return fail(FW_ERR_INVALID, "warp mask: the product image is not on the grid of the field");
    fw_image* im = product;
    if (!im) FW_TRY(new_image(ctx, field->grid, &im));
    int rc = launch_warp(ctx, mask, field, pre, affine, im->d, true, product ? product->d : nullptr);
    if (!rc) rc = sync(ctx);
    if (rc) {
        if (!product) fw_image_free(im);
        return rc;
    }
    *out = im;
    return 0;
}

int fw_max_scaled_norm(fw_ctx* ctx, const fw_field* field, double* out) {
    FW_CHECK(ctx && field && out, "null argument");
    unsigned int* bits = ctx->d_counter + 32;
    FW_CUDA(cudaMemsetAsync(bits, 0, sizeof(unsigned int), ctx->stream));
    FW_TRY(launch_max_norm(ctx, field, bits));
    unsigned int h = 0;
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, bits, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    FW_TRY(sync(ctx));
    std::memcpy(&h, ctx->h_pinned, sizeof(h));
    float f;
    std::memcpy(&f, &h, sizeof(f));
    *out = std::isnan(f) ? NAN : (double)f;
    return 0;
}

int fw_max_scaled_norm_pair(fw_ctx* ctx, const fw_field* a, const fw_field* b, double out[2]) {
    FW_CHECK(ctx && a && b && out, "null argument");
    unsigned int* bits = ctx->d_counter + 32;
    FW_CUDA(cudaMemsetAsync(bits, 0, 2 * sizeof(unsigned int), ctx->stream));
    FW_TRY(launch_max_norm(ctx, a, bits));
    FW_TRY(launch_max_norm(ctx, b, bits + 1));
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, bits, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    FW_TRY(sync(ctx));
    unsigned int h[2];
    std::memcpy(h, ctx->h_pinned, sizeof(h));
    for (int i = 0; i < 2; ++i) {
        float f;
        std::memcpy(&f, &h[i], sizeof(f));
        out[i] = std::isnan(f) ? NAN : (double)f;
    }
    return 0;
}

int fw_l2_norm(fw_ctx* ctx, const fw_field* field, double* out) {
    FW_CHECK(ctx && field && out, "null argument");
    FW_TRY(reduce_l2(ctx, field, ctx->d_scratch + SLOT_NORM_A));
    double s;
    FW_TRY(read_scalars(ctx, ctx->d_scratch + SLOT_NORM_A, 1, &s));
    *out = std::sqrt(s);
    return 0;
}

int fw_scale(fw_ctx* ctx, fw_field* field, double s) {
    FW_CHECK(ctx && field, "null argument");
    long long n4 = 3 * field->ps / 4;
    k_scale<<<(unsigned)((n4 + 255) / 256), 256, 0, ctx->stream>>>((float4*)field->d, n4, (float)s);
    FW_TRY(check_launch(ctx, "k_scale"));
    return sync(ctx);
}

int fw_axpy(fw_ctx* ctx, fw_field* acc, double a, const fw_field* x) {
    FW_CHECK(ctx && acc && x, "null argument");
    if (!acc->grid.same(x->grid)) return fail(FW_ERR_INVALID, "field axpy: grids differ");
    long long n4 = 3 * acc->ps / 4;
    k_axpy<<<(unsigned)((n4 + 255) / 256), 256, 0, ctx->stream>>>((float4*)acc->d, (const float4*)x->d, n4, (float)a);
    FW_TRY(check_launch(ctx, "k_axpy"));
    return sync(ctx);
}

int fw_compose(fw_ctx* ctx, const fw_field* displacement, const fw_field* warping, fw_field** out) {
    FW_CHECK(ctx && displacement && warping && out, "null argument");
    if (!displacement->grid.same(warping->grid))
        return fail(FW_ERR_INVALID, "compose: displacement and warping grids differ");
    fw_field* f;
    FW_TRY(new_field(ctx, warping->grid, &f));
    int rc = launch_compose(ctx, displacement, warping, f, nullptr, 1.0);
    if (!rc) rc = sync(ctx);
    if (rc) {
        fw_field_free(f);
        return rc;
    }
    *out = f;
    return 0;
}

int fw_resample_field(fw_ctx* ctx, const fw_field* field, const fw_grid* grid, fw_field** out) {
    FW_CHECK(ctx && field && grid && out, "null argument");
    HostGrid g;
    FW_TRY(make_grid(grid, g));
    if (g.same(field->grid)) return fw_field_copy(ctx, field, out);
    fw_field* f;
    FW_TRY(new_field(ctx, g, &f));
    int rc = launch_resample(ctx, field, f);
    if (!rc) rc = sync(ctx);
    if (rc) {
        fw_field_free(f);
        return rc;
    }
    *out = f;
    return 0;
}

}  // extern "C"
