// fw_samples.cu -- a linear stage level's Mattes MI samples, prepared on the device, and the
// centre of mass of an image.
//
// The reference draws and prepares a level's samples on the host (sampling.rs:181-238,
// linear.rs:251-280, 474-492, 940-945, metric/mi.rs:121-317). Here the host only draws the
// MT19937 integers (a sequential generator, six per sample point), on host threads started when
// a stage begins, one per level, so that they overlap the earlier levels; the context keeps the
// uploaded integers by (seed, picks) for the next registration of the same level grid. The rest
// is four kernels:
//   pick     one thread per raster pick: the jittered point (ITK's Box-Muller variate), the
//            fixed-mask test, the nearest fixed voxel's value (the fixed range) and the trilinear
//            fixed value (whether the point is kept); per block the counts, the extreme keys and
//            the kept points' coordinate sums;
//   mrange   the smoothed moving image's finite range (order-preserving keys, atomics);
//   scan     one block: the blocks' output offsets and the totals, the cloud centre summed in a
//            fixed order;
//   records  after the host has formed the binning from the ranges, the kept points' records
//            (float32 offsets from the centre, the fixed bin) in raster order.
// Only a small summary comes back to the host. Every point, index map and interpolation follows
// the host restatement's float64 operation order with no fused multiply-adds; the variate calls
// the device's log and cos, which may differ from the host library's in the last bit.
#include "fw_internal.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <future>
#include <string>
#include <vector>

namespace fw {
namespace {

constexpr int SP_THREADS = 256;
constexpr int SCAN_THREADS = 1024;

// MT19937 (Matsumoto & Nishimura 1998) with the reference's seeding (sampling.rs:40-120).
struct Mt19937 {
    uint32_t s[624];
    int next = 0, left = 0;
    static uint32_t twist(uint32_t m, uint32_t s0, uint32_t s1) {
        return m ^ (((s0 & 0x80000000u) | (s1 & 0x7fffffffu)) >> 1) ^ ((s1 & 1u) ? 0x9908b0dfu : 0u);
    }
    explicit Mt19937(uint32_t seed) {
        s[0] = seed;
        for (uint32_t i = 1; i < 624; ++i) s[i] = 1812433253u * (s[i - 1] ^ (s[i - 1] >> 30)) + i;
        reload();
    }
    void reload() {
        for (int p = 0; p < 624; ++p) s[p] = twist(s[(p + 397) % 624], s[p], s[(p + 1) % 624]);
        left = 624;
        next = 0;
    }
    uint32_t integer() {
        if (left == 0) reload();
        --left;
        uint32_t y = s[next++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        return y ^ (y >> 18);
    }
};

__device__ __forceinline__ unsigned int value_key(float v) {
    const unsigned int b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__host__ __device__ __forceinline__ float key_float(unsigned int k) {
#ifdef __CUDA_ARCH__
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
#else
    const unsigned int b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
#endif
}

struct PickArgs {
    DevGrid lg;             // the level grid: the sample raster
    DevGrid fg;             // the fixed image's grid
    DevGrid kg;             // the fixed mask's grid (when masked)
    const uint32_t* draws;  // six MT19937 integers per pick
    long long picks, stride;
    double jit[3];          // the level grid's spacing / 3 per axis (the jitter's deviation)
    const float* fixed;     // the level's smoothed fixed image
    const float* mask;      // nullable
    unsigned char* flags;   // per pick: 1 inside the mask, 2 on a finite nearest voxel, 4 kept
    unsigned int* counts;   // [3][blocks]: inside the mask, on a finite nearest voxel, kept
    double* sums;           // [blocks][3]: the kept points' coordinate sums
    unsigned int* keys;     // [4]: fixed min / max, moving min / max (order-preserving keys)
};

// sampling.rs:163-171: ITK's Box-Muller variate (cosine branch) from two integer draws.
__device__ __forceinline__ double normal_from(uint32_t open, uint32_t open_upper) {
    const double o = __dmul_rn(__dadd_rn((double)open, 0.5), 1.0 / 4294967296.0);
    const double ou = __dmul_rn((double)open_upper, 1.0 / 4294967296.0);
    const double r = sqrt(__dmul_rn(__dmul_rn(-2.0, log(__dsub_rn(1.0, o))), 1.0));
    return __dmul_rn(r, cos(__dmul_rn(2.0 * M_PI, ou)));
}

// sampling.rs:196-238: pick q is voxel q * stride in raster order, jittered by N(0, 1) *
// spacing / 3 per axis (two draws per variate, x first).
__device__ __forceinline__ void pick_point(const PickArgs& a, long long q, double p[3]) {
    const long long flat = q * a.stride;
    const long long nx = a.lg.nx, ny = a.lg.ny;
    exact_point(a.lg, (double)(flat % nx), (double)((flat / nx) % ny), (double)(flat / (nx * ny)), p);
    const uint32_t* d = a.draws + 6 * q;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
        p[ax] = __dadd_rn(p[ax], __dmul_rn(normal_from(__ldg(d + 2 * ax), __ldg(d + 2 * ax + 1)), a.jit[ax]));
}

// The nearest voxel (rounding half up) of continuous index c, when inside the buffer.
__device__ __forceinline__ bool nearest_voxel(const DevGrid& g, const double c[3], long long& off) {
    const int n[3] = {g.nx, g.ny, g.nz};
    long long q[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const double r = floor(__dadd_rn(c[ax], 0.5));
        if (!(r >= 0.0 && r < (double)n[ax])) return false;
        q[ax] = (long long)r;
    }
    off = q[0] + (long long)g.nx * (q[1] + (long long)g.ny * q[2]);
    return true;
}

// mask.rs:76-110 (MaskVolume::is_inside): the mask's nearest voxel is inside and not zero.
__device__ __forceinline__ bool mask_inside(const DevGrid& g, const float* m, const double p[3]) {
    double c[3];
    exact_index(g, p, c);
    long long off;
    return nearest_voxel(g, c, off) && __ldg(m + off) != 0.0f;
}

// interp.rs:43-85 in float64 over a float32 image: ITK's linear interpolation at a continuous
// index inside the buffer ([-0.5, n - 0.5) per axis), neighbours clamped, the host
// restatement's operation order.
__device__ __forceinline__ bool lin_f64(const DevGrid& g, const float* img, const double c[3],
                                        double& out) {
    const int n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
        if (!(c[ax] >= -0.5 && c[ax] < (double)n[ax] - 0.5)) return false;
    long long b[3];
    double w[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const double fl = floor(c[ax]);
        double d;
        if (fl < 0.0) {
            b[ax] = 0;
            d = c[ax];
        } else if (!(fl <= (double)(n[ax] - 1))) {
            b[ax] = n[ax] - 1;
            d = __dsub_rn(c[ax], (double)(n[ax] - 1));
        } else {
            b[ax] = (long long)fl;
            d = __dsub_rn(c[ax], fl);
        }
        w[ax] = (d <= 0.0 || b[ax] + 1 > n[ax] - 1) ? 0.0 : d;
    }
    const long long sy = g.nx, sz = (long long)g.nx * g.ny;
    const long long base = b[0] + sy * b[1] + sz * b[2];
    const long long ox = w[0] > 0.0 ? 1 : 0, oy = w[1] > 0.0 ? sy : 0, oz = w[2] > 0.0 ? sz : 0;
    auto at = [&](long long o) { return (double)__ldg(img + base + o); };
    auto plane = [&](long long o) {
        const double v00 = at(o), v10 = at(o + ox), v01 = at(o + oy), v11 = at(o + oy + ox);
        const double x0 = __dadd_rn(v00, __dmul_rn(__dsub_rn(v10, v00), w[0]));
        const double x1 = __dadd_rn(v01, __dmul_rn(__dsub_rn(v11, v01), w[0]));
        return __dadd_rn(x0, __dmul_rn(__dsub_rn(x1, x0), w[1]));
    };
    const double y0 = plane(0);
    out = w[2] > 0.0 ? __dadd_rn(y0, __dmul_rn(__dsub_rn(plane(oz), y0), w[2])) : y0;
    return true;
}

__global__ void __launch_bounds__(SP_THREADS) k_samples_pick(const PickArgs a) {
    const long long q = (long long)blockIdx.x * SP_THREADS + threadIdx.x;
    unsigned int inside = 0, seen = 0, kept = 0, klo = 0xffffffffu, khi = 0u;
    double p[3] = {0.0, 0.0, 0.0};
    if (q < a.picks) {
        pick_point(a, q, p);
        if (!a.mask || mask_inside(a.kg, a.mask, p)) {
            inside = 1;
            double c[3];
            exact_index(a.fg, p, c);
            long long off;
            if (nearest_voxel(a.fg, c, off)) {
                const float v = __ldg(a.fixed + off);
                if (isfinite(v)) {
                    seen = 1;
                    klo = khi = value_key(v);
                }
            }
            double f;
            if (lin_f64(a.fg, a.fixed, c, f) && isfinite(f)) kept = 1;
        }
        a.flags[q] = (unsigned char)(inside | (seen << 1) | (kept << 2));
    }
    if (!kept) p[0] = p[1] = p[2] = 0.0;
    __shared__ unsigned int scnt[3][SP_THREADS / 32], skey[2][SP_THREADS / 32];
    __shared__ double ssum[3][SP_THREADS / 32];
    const unsigned int full = 0xffffffffu;
    const unsigned int c0 = __reduce_add_sync(full, inside), c1 = __reduce_add_sync(full, seen),
                       c2 = __reduce_add_sync(full, kept);
    const unsigned int k0 = __reduce_min_sync(full, klo), k1 = __reduce_max_sync(full, khi);
    double s[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) s[ax] = warp_sum_d(p[ax]);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        scnt[0][w] = c0;
        scnt[1][w] = c1;
        scnt[2][w] = c2;
        skey[0][w] = k0;
        skey[1][w] = k1;
        for (int ax = 0; ax < 3; ++ax) ssum[ax][w] = s[ax];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t0 = 0, t1 = 0, t2 = 0, lo = 0xffffffffu, hi = 0u;
        double u[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < SP_THREADS / 32; ++k) {
            t0 += scnt[0][k];
            t1 += scnt[1][k];
            t2 += scnt[2][k];
            lo = min(lo, skey[0][k]);
            hi = max(hi, skey[1][k]);
            for (int ax = 0; ax < 3; ++ax) u[ax] += ssum[ax][k];
        }
        const long long nb = gridDim.x;
        a.counts[blockIdx.x] = t0;
        a.counts[nb + blockIdx.x] = t1;
        a.counts[2 * nb + blockIdx.x] = t2;
        for (int ax = 0; ax < 3; ++ax) a.sums[3 * (long long)blockIdx.x + ax] = u[ax];
        if (t1) {
            atomicMin(a.keys, lo);
            atomicMax(a.keys + 1, hi);
        }
    }
}

// metric/mi.rs:229-262 (MiBinning::new, moving side): the finite range of the whole image.
__global__ void __launch_bounds__(SP_THREADS) k_samples_mrange(const float* __restrict__ m,
                                                                long long n,
                                                                unsigned int* keys) {
    unsigned int lo = 0xffffffffu, hi = 0u;
    const long long stride = (long long)gridDim.x * SP_THREADS;
    for (long long l = (long long)blockIdx.x * SP_THREADS + threadIdx.x; l < n; l += stride) {
        const float v = __ldg(m + l);
        if (isfinite(v)) {
            const unsigned int k = value_key(v);
            lo = min(lo, k);
            hi = max(hi, k);
        }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if ((threadIdx.x & 31) == 0 && hi != 0u) {
        atomicMin(keys + 2, lo);
        atomicMax(keys + 3, hi);
    }
}

struct SampleSummary {
    unsigned long long inside, seen, kept;
    unsigned int keys[4];
    double sum[3];  // the kept points' coordinate sums
};

// One block: exclusive offsets of the blocks' kept counts, the totals, and the coordinate sums
// over the blocks in a fixed order.
__global__ void __launch_bounds__(SCAN_THREADS) k_samples_scan(const unsigned int* counts,
                                                               int nb, const double* sums,
                                                               const unsigned int* keys,
                                                               unsigned long long* offsets,
                                                               SampleSummary* out) {
    __shared__ unsigned long long scan[SCAN_THREADS];
    __shared__ unsigned long long tot[2][SCAN_THREADS / 32];
    __shared__ double red[SCAN_THREADS / 32];
    const int t = threadIdx.x;
    const int per = (nb + SCAN_THREADS - 1) / SCAN_THREADS;
    const int lo = min(t * per, nb), hi = min(lo + per, nb);
    unsigned long long c0 = 0, c1 = 0, c2 = 0;
    for (int k = lo; k < hi; ++k) {
        c0 += counts[k];
        c1 += counts[nb + k];
        c2 += counts[2 * nb + k];
    }
    scan[t] = c2;
    __syncthreads();
    for (int o = 1; o < SCAN_THREADS; o <<= 1) {
        const unsigned long long v = t >= o ? scan[t - o] : 0ull;
        __syncthreads();
        scan[t] += v;
        __syncthreads();
    }
    unsigned long long base = scan[t] - c2;
    for (int k = lo; k < hi; ++k) {
        offsets[k] = base;
        base += counts[2 * nb + k];
    }
    for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_xor_sync(0xffffffffu, c0, o);
        c1 += __shfl_xor_sync(0xffffffffu, c1, o);
    }
    if ((t & 31) == 0) {
        tot[0][t >> 5] = c0;
        tot[1][t >> 5] = c1;
    }
    __syncthreads();
    double s[3];
    for (int ax = 0; ax < 3; ++ax) s[ax] = block_sum_fixed(sums + ax, (unsigned int)nb, 3, red);
    if (t == 0) {
        unsigned long long a0 = 0, a1 = 0;
        for (int w = 0; w < SCAN_THREADS / 32; ++w) {
            a0 += tot[0][w];
            a1 += tot[1][w];
        }
        out->inside = a0;
        out->seen = a1;
        out->kept = scan[SCAN_THREADS - 1];
        for (int k = 0; k < 4; ++k) out->keys[k] = keys[k];
        for (int ax = 0; ax < 3; ++ax) out->sum[ax] = s[ax];
    }
}

struct RecordArgs {
    double center[3];
    double fixed_bin_size, fixed_normalized_min;
    int bins;
};

// prepare_samples (linear.rs:251-280): each kept point's record, in raster order: its offset
// from the cloud centre in float32 and its fixed bin (the trilinear value's box-window bin,
// metric/mi.rs:121-155, clamped to [2, bins - 3]).
__global__ void __launch_bounds__(SP_THREADS) k_samples_records(const PickArgs a,
                                                                const unsigned long long* offsets,
                                                                const RecordArgs r, float4* rec) {
    const long long q = (long long)blockIdx.x * SP_THREADS + threadIdx.x;
    const bool kept = q < a.picks && (a.flags[q] & 4u);
    const unsigned int ballot = __ballot_sync(0xffffffffu, kept);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __shared__ unsigned int wbase[SP_THREADS / 32];
    if (lane == 0) wbase[w] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int acc = 0;
        for (int k = 0; k < SP_THREADS / 32; ++k) {
            const unsigned int c = wbase[k];
            wbase[k] = acc;
            acc += c;
        }
    }
    __syncthreads();
    if (!kept) return;
    double p[3], c[3], f = 0.0;
    pick_point(a, q, p);
    exact_index(a.fg, p, c);
    lin_f64(a.fg, a.fixed, c, f);
    const double term = __dsub_rn(__ddiv_rn(f, r.fixed_bin_size), r.fixed_normalized_min);
    long long idx = isnan(term) ? 0 : (long long)term;
    idx = idx < 2 ? 2 : (idx > r.bins - 3 ? r.bins - 3 : idx);
    const unsigned long long at =
        offsets[blockIdx.x] + wbase[w] + __popc(ballot & ((1u << lane) - 1u));
    rec[at] = make_float4(__double2float_rn(__dsub_rn(p[0], r.center[0])),
                          __double2float_rn(__dsub_rn(p[1], r.center[1])),
                          __double2float_rn(__dsub_rn(p[2], r.center[2])),
                          __uint_as_float((unsigned int)idx));
}

// init.rs:50-74 (centre_of_gravity): per block the mass and the intensity-weighted sums of the
// voxel centres over a contiguous raster range, float64.
__global__ void __launch_bounds__(SP_THREADS) k_com_partials(const float* __restrict__ img,
                                                             const DevGrid g, long long chunk,
                                                             double* part) {
    const long long n = g.n;
    const long long lo = (long long)blockIdx.x * chunk, hi = min(lo + chunk, n);
    double m = 0.0, s[3] = {0.0, 0.0, 0.0};
    for (long long l = lo + threadIdx.x; l < hi; l += SP_THREADS) {
        const double v = (double)__ldg(img + l);
        double p[3];
        exact_point(g, (double)(l % g.nx), (double)((l / g.nx) % g.ny), (double)(l / ((long long)g.nx * g.ny)), p);
        m = __dadd_rn(m, v);
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) s[ax] = __dadd_rn(s[ax], __dmul_rn(p[ax], v));
    }
    __shared__ double red[4][SP_THREADS / 32];
    const double r[4] = {warp_sum_d(m), warp_sum_d(s[0]), warp_sum_d(s[1]), warp_sum_d(s[2])};
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 4; ++k) red[k][threadIdx.x >> 5] = r[k];
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int w = 0; w < SP_THREADS / 32; ++w) t += red[threadIdx.x][w];
        part[4 * (long long)blockIdx.x + threadIdx.x] = t;
    }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_com_finish(const double* part, int nb,
                                                             double* out) {
    __shared__ double red[SCAN_THREADS / 32];
    for (int k = 0; k < 4; ++k) {
        const double s = block_sum_fixed(part + k, (unsigned int)nb, 4, red);
        if (threadIdx.x == 0) out[k] = s;
    }
}

__global__ void __launch_bounds__(SP_THREADS) k_any_nonzero(const float* __restrict__ m,
                                                            long long n, unsigned int* flag) {
    const long long stride = (long long)gridDim.x * SP_THREADS;
    unsigned int any = 0;
    for (long long l = (long long)blockIdx.x * SP_THREADS + threadIdx.x; l < n; l += stride)
        any |= __ldg(m + l) != 0.0f;
    any = __reduce_or_sync(0xffffffffu, any);
    if ((threadIdx.x & 31) == 0 && any) atomicOr(flag, 1u);
}

unsigned int stream_blocks(const fw_ctx* ctx, long long n) {
    const long long want = (n + SP_THREADS - 1) / SP_THREADS;
    return (unsigned int)std::max<long long>(1, std::min<long long>(want, 8LL * ctx->num_sms));
}

// Device buffers of one preparation, freed together.
struct Scratch {
    fw_ctx* ctx;
    std::vector<std::pair<void*, size_t>> held;
    explicit Scratch(fw_ctx* c) : ctx(c) {}
    template <typename T>
    int get(size_t count, T** out) {
        const size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
        void* p = nullptr;
        FW_TRY(dev_alloc(ctx, bytes, &p));
        held.emplace_back(p, bytes);
        *out = static_cast<T*>(p);
        return 0;
    }
    ~Scratch() {
        for (auto& h : held) dev_free(ctx, h.first, h.second);
    }
};

long long level_stride(float percentage) {
    return (long long)std::max(std::ceil(1.0 / (double)percentage), 1.0);
}

std::vector<uint32_t> generate_draws(uint32_t seed, long long picks) {
    std::vector<uint32_t> v(6 * (size_t)picks);
    Mt19937 mt(seed);
    for (auto& x : v) x = mt.integer();
    return v;
}

constexpr size_t MAX_DRAW_BUFFERS = 8;
constexpr size_t MAX_DRAW_BYTES = (size_t)1 << 30;

// The device copy of the draws of (seed, picks): the context's kept copy, or the plan's
// generated ones, or generated here, uploaded and kept.
int level_draws(fw_ctx* ctx, uint32_t seed, long long picks, DrawPlan* plan, const uint32_t** out) {
    for (auto& e : ctx->draws)
        if (e.seed == seed && e.picks == picks) {
            e.used = ++ctx->draws_tick;
            *out = e.d;
            return 0;
        }
    const size_t count = 6 * (size_t)picks, bytes = sizeof(uint32_t) * count;
    // make room: at most MAX_DRAW_BUFFERS copies and MAX_DRAW_BYTES, the least recently used out
    size_t held = bytes;
    for (auto& e : ctx->draws) held += e.bytes;
    while (!ctx->draws.empty() &&
           (ctx->draws.size() >= MAX_DRAW_BUFFERS || held > MAX_DRAW_BYTES)) {
        auto lru = std::min_element(ctx->draws.begin(), ctx->draws.end(),
                                    [](const fw_ctx::DrawBuffer& a, const fw_ctx::DrawBuffer& b) {
                                        return a.used < b.used;
                                    });
        held -= lru->bytes;
        dev_free(ctx, lru->d, lru->bytes);
        ctx->draws.erase(lru);
    }
    uint32_t* d = nullptr;
    FW_TRY(dev_alloc(ctx, bytes, (void**)&d));
    std::vector<uint32_t> pre;
    if (plan)
        for (auto& j : plan->jobs)
            if (j.seed == seed && j.picks == picks && j.draws.valid()) {
                pre = j.draws.get();
                break;
            }
    cudaError_t e;
    if (pre.size() == count) {
        // pageable: the copy has left `pre` when the call returns
        e = cudaMemcpyAsync(d, pre.data(), bytes, cudaMemcpyHostToDevice, ctx->stream);
    } else {
        uint32_t* h = nullptr;
        int rc = host_stage(ctx, bytes, (void**)&h);
        if (rc) {
            dev_free(ctx, d, bytes);
            return rc;
        }
        Mt19937 mt(seed);
        for (size_t k = 0; k < count; ++k) h[k] = mt.integer();
        // the staging buffer is written again only after the caller's next synchronisation
        e = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ctx->stream);
    }
    if (e != cudaSuccess) {
        dev_free(ctx, d, bytes);
        return cuda_fail(e, "sample draws upload");
    }
    ctx->stats.bytes_uploaded += bytes;
    ctx->draws.push_back(fw_ctx::DrawBuffer{seed, (int64_t)picks, d, bytes, ++ctx->draws_tick});
    *out = d;
    return 0;
}

}  // namespace

void plan_draws(fw_ctx* ctx, DrawPlan& plan, const HostGrid& lg, float percentage, uint32_t seed) {
    const long long stride = level_stride(percentage);
    const long long picks = (lg.count() + stride - 1) / stride;
    for (auto& e : ctx->draws)
        if (e.seed == seed && e.picks == picks) return;
    for (auto& j : plan.jobs)
        if (j.seed == seed && j.picks == picks) return;
    plan.jobs.push_back(DrawPlan::Job{seed, (int64_t)picks,
                                      std::async(std::launch::async, generate_draws, seed, picks)});
}

void drop_draws(fw_ctx* ctx) {
    for (auto& e : ctx->draws) dev_free(ctx, e.d, e.bytes);
    ctx->draws.clear();
}

int mask_has_inside(fw_ctx* ctx, const fw_image* mask, bool* any) {
    Scratch sc(ctx);
    unsigned int* flag;
    FW_TRY(sc.get(1, &flag));
    FW_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned int), ctx->stream));
    const long long n = mask->grid.count();
    k_any_nonzero<<<stream_blocks(ctx, n), SP_THREADS, 0, ctx->stream>>>(mask->d, n, flag);
    FW_TRY(check_launch(ctx, "k_any_nonzero"));
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, flag, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    FW_TRY(sync(ctx));
    unsigned int h;
    std::memcpy(&h, ctx->h_pinned, sizeof(h));
    *any = h != 0;
    return 0;
}

int centre_of_mass(fw_ctx* ctx, const fw_image* img, double out[3]) {
    const HostGrid& g = img->grid;
    const long long n = g.count();
    const int nb = (int)std::max<long long>(1, std::min<long long>(4LL * ctx->num_sms, (n + 1023) / 1024));
    const long long chunk = (n + nb - 1) / nb;
    Scratch sc(ctx);
    double *part, *res;
    FW_TRY(sc.get(4 * (size_t)nb, &part));
    FW_TRY(sc.get(4, &res));
    k_com_partials<<<nb, SP_THREADS, 0, ctx->stream>>>(img->d, dev_grid(g), chunk, part);
    FW_TRY(check_launch(ctx, "k_com_partials"));
    k_com_finish<<<1, SCAN_THREADS, 0, ctx->stream>>>(part, nb, res);
    FW_TRY(check_launch(ctx, "k_com_finish"));
    double h[4];
    FW_TRY(read_back(ctx, res, 4, h));
    if (h[0] == 0.0) return fail(FW_ERR_INVALID, "total mass of the image is zero");
    for (int a = 0; a < 3; ++a) out[a] = h[1 + a] / h[0];
    return 0;
}

int prepare_level_samples(fw_ctx* ctx, const HostGrid& lg, const fw_image* fixed,
                          const fw_image* moving, const fw_image* mask, float percentage,
                          uint32_t seed, int bins, LevelSamples& out, DrawPlan* plan) {
    out = LevelSamples{};
    const long long stride = level_stride(percentage);
    const long long picks = (lg.count() + stride - 1) / stride;
    const long long nbl = (picks + SP_THREADS - 1) / SP_THREADS;
    FW_CHECK(nbl < (1LL << 31), "linear stage: too many sample points for one level");
    const int nb = (int)nbl;
    // the six integer draws of every pick, in the generator's order
    const uint32_t* draws = nullptr;
    FW_TRY(level_draws(ctx, seed, picks, plan, &draws));
    Scratch sc(ctx);
    unsigned char* flags;
    unsigned int *counts, *keys;
    double* sums;
    unsigned long long* offsets;
    SampleSummary* summary;
    FW_TRY(sc.get((size_t)picks, &flags));
    FW_TRY(sc.get(3 * (size_t)nb, &counts));
    FW_TRY(sc.get(4, &keys));
    FW_TRY(sc.get(3 * (size_t)nb, &sums));
    FW_TRY(sc.get((size_t)nb, &offsets));
    FW_TRY(sc.get(1, &summary));
    const unsigned int init[4] = {0xffffffffu, 0u, 0xffffffffu, 0u};
    FW_CUDA(cudaMemcpyAsync(keys, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
    PickArgs a{};
    a.lg = dev_grid(lg);
    a.fg = dev_grid(fixed->grid);
    if (mask) a.kg = dev_grid(mask->grid);
    a.draws = draws;
    a.picks = picks;
    a.stride = stride;
    for (int ax = 0; ax < 3; ++ax) a.jit[ax] = lg.sp[ax] / 3.0;
    a.fixed = fixed->d;
    a.mask = mask ? mask->d : nullptr;
    a.flags = flags;
    a.counts = counts;
    a.sums = sums;
    a.keys = keys;
    k_samples_pick<<<nb, SP_THREADS, 0, ctx->stream>>>(a);
    FW_TRY(check_launch(ctx, "k_samples_pick"));
    const long long nm = moving->grid.count();
    k_samples_mrange<<<stream_blocks(ctx, nm), SP_THREADS, 0, ctx->stream>>>(moving->d, nm, keys);
    FW_TRY(check_launch(ctx, "k_samples_mrange"));
    k_samples_scan<<<1, SCAN_THREADS, 0, ctx->stream>>>(counts, nb, sums, keys, offsets, summary);
    FW_TRY(check_launch(ctx, "k_samples_scan"));
    FW_CUDA(cudaMemcpyAsync(ctx->h_pinned, summary, sizeof(SampleSummary), cudaMemcpyDeviceToHost,
                            ctx->stream));
    FW_TRY(sync(ctx));  // also ends any upload of the draws: the staging buffer is free again
    SampleSummary h;
    std::memcpy(&h, ctx->h_pinned, sizeof(h));
    out.candidates = (int64_t)h.inside;
    char msg[256];
    // linear.rs:474-492: a level whose samples leave Mattes MI undefined is skipped
    if (h.seen == 0) {
        std::snprintf(msg, sizeof(msg), "no sample point lands on the fixed image inside the fixed "
                      "mask, if one is given (%lld candidate points on the level grid)",
                      (long long)h.inside);
        out.skip = true;
        out.why = msg;
        return 0;
    }
    const double lo = (double)key_float(h.keys[0]), hi = (double)key_float(h.keys[1]);
    if (hi - lo <= DBL_EPSILON) {
        std::snprintf(msg, sizeof(msg), "the fixed image takes a single value at its %lld sample "
                      "point(s) (%lld candidate points)", (long long)h.seen, (long long)h.inside);
        out.skip = true;
        out.why = msg;
        return 0;
    }
    if (h.keys[3] == 0u) return fail(FW_ERR_INVALID, "the moving image has no finite voxel");
    const double mlo = (double)key_float(h.keys[2]), mhi = (double)key_float(h.keys[3]);
    if (mhi - mlo <= DBL_EPSILON) return fail(FW_ERR_INVALID, "the moving image is constant");
    // MiBinning::new (metric/mi.rs:229-262)
    fw_mi_binning& b = out.binning;
    const double span = (double)(bins - 4);
    b.bins = bins;
    b.fixed_min = lo;
    b.fixed_max = hi;
    b.moving_min = mlo;
    b.moving_max = mhi;
    b.fixed_bin_size = (hi - lo) / span;
    b.moving_bin_size = (mhi - mlo) / span;
    b.fixed_normalized_min = lo / b.fixed_bin_size - 2.0;
    b.moving_normalized_min = mlo / b.moving_bin_size - 2.0;
    if (h.kept == 0) {
        std::snprintf(msg, sizeof(msg), "no sample point lies inside the fixed image (%lld "
                      "candidate points)", (long long)h.inside);
        out.skip = true;
        out.why = msg;
        return 0;
    }
    out.n = (int64_t)h.kept;
    for (int ax = 0; ax < 3; ++ax) out.center[ax] = h.sum[ax] / (double)out.n;
    FW_TRY(dev_alloc(ctx, sizeof(float4) * (size_t)out.n, (void**)&out.d_rec));
    RecordArgs r{};
    for (int ax = 0; ax < 3; ++ax) r.center[ax] = out.center[ax];
    r.fixed_bin_size = b.fixed_bin_size;
    r.fixed_normalized_min = b.fixed_normalized_min;
    r.bins = bins;
    k_samples_records<<<nb, SP_THREADS, 0, ctx->stream>>>(a, offsets, r, out.d_rec);
    int rc = check_launch(ctx, "k_samples_records");
    if (rc) {
        dev_free(ctx, out.d_rec, sizeof(float4) * (size_t)out.n);
        out.d_rec = nullptr;
    }
    return rc;
}

void free_level_samples(fw_ctx* ctx, LevelSamples& s) {
    if (s.d_rec) dev_free(ctx, s.d_rec, sizeof(float4) * (size_t)s.n);
    s.d_rec = nullptr;
}

}  // namespace fw
