// gen.cu -- seeded droplet generator with overlap rejection on the device.
//
// The reference's UniformDropletGenerator (dem/particle_generator/
// uniform_droplet_generator.py:45-164) draws radii and positions uniformly and
// then, round after round, re-draws every droplet still listed as overlapping
// and lists again those of the re-drawn droplets that overlap any droplet
// (distance < r_i + r_j + minimum_distance), until none is listed or 1,000
// rounds have passed.  Here a round is:
//
//   1. draw the listed droplets' positions (all droplets in round 0);
//   2. find every overlapping pair with the spatial hash (csrc/hash.cu) on
//      radii inflated by minimum_distance / 2, so that d <= r'_i + r'_j is
//      d <= r_i + r_j + minimum_distance (the reference's strict < differs only
//      on the boundary); in a periodic box the hash uses whole cells, so pairs
//      touching across the periodic faces are found as well;
//   3. list the droplets that were just drawn and belong to such a pair.
//
// Random numbers are a counter-based stream: SplitMix64 (Steele, Lea and
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014) of
// (seed, purpose, round, droplet), so a seed fixes the state independently of
// the launch shape.  Positions are drawn in [0, hi - lo) and shifted at the end.
#include <cmath>

#include "common.cuh"

namespace dem {
int launch_hash_detect(dem_ctx *, int, const double *, const double *, const double *, const double *, double, int,
                       int, int32_t *, int64_t, int64_t *, cudaStream_t, int);
}

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// uniform in [0, 1) with 53 random bits
__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t stream, uint64_t idx) {
    const uint64_t u = splitmix64(splitmix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) + idx);
    return (double)(u >> 11) * 0x1.0p-53;
}

constexpr uint64_t STREAM_RADII = 1;
__device__ __forceinline__ uint64_t stream_pos(int round, int axis) { return 2 + 3 * (uint64_t)round + axis; }

__global__ void draw_radii_kernel(int n, uint64_t seed, double rmin, double rmax, double half_gap,
                                  double *__restrict__ r, double *__restrict__ rr) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = rmin + (rmax - rmin) * uniform01(seed, STREAM_RADII, i);
        r[i] = v;
        rr[i] = v + half_gap;
    }
}

// round 0 draws every droplet (listed == NULL)
__global__ void draw_positions_kernel(int n, uint64_t seed, int round, double span, const int32_t *__restrict__ listed,
                                      double *__restrict__ x, double *__restrict__ y, double *__restrict__ z) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (listed && !listed[i]) continue;
        x[i] = span * uniform01(seed, stream_pos(round, 0), i);
        y[i] = span * uniform01(seed, stream_pos(round, 1), i);
        z[i] = span * uniform01(seed, stream_pos(round, 2), i);
    }
}

// next[i] = 1 for every just-drawn droplet (drawn[i], or all when drawn == NULL)
// that belongs to an overlapping pair; count = number of such droplets
__global__ void flag_overlaps_kernel(const int32_t *__restrict__ pairs, const int64_t *__restrict__ counts,
                                     const int32_t *__restrict__ drawn, int32_t *__restrict__ next,
                                     unsigned long long *__restrict__ listed_count) {
    const int64_t k = counts[0];
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < k; p += (int64_t)gridDim.x * blockDim.x) {
        const int i = pairs[2 * p], j = pairs[2 * p + 1];
        if ((!drawn || drawn[i]) && atomicExch(&next[i], 1) == 0) atomicAdd(listed_count, 1ull);
        if ((!drawn || drawn[j]) && atomicExch(&next[j], 1) == 0) atomicAdd(listed_count, 1ull);
    }
}

__global__ void shift_kernel(int n, double lo, double *__restrict__ x, double *__restrict__ y,
                             double *__restrict__ z) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] += lo;
        y[i] += lo;
        z[i] += lo;
    }
}

int next_pow2(int64_t v) {
    int64_t p = 1;
    while (p < v) p <<= 1;
    return (int)p;
}

}  // namespace

extern "C" {

int dem_generate_droplets(dem_ctx *ctx, int n, unsigned long long seed, double lo, double hi, double rmin,
                          double rmax, double minimum_distance, int periodic, int max_rounds, double *x, double *y,
                          double *z, double *r, int *rounds_out, void *stream) {
    if (!ctx) return DEM_E_INVALID;
    if (n < 0) return dem_set_error(ctx, DEM_E_INVALID, "n must be >= 0");
    if (n > ctx->capacity) return dem_set_error(ctx, DEM_E_CAPACITY, "number of droplets exceeds the capacity");
    if (!(hi > lo) || !(rmax >= rmin) || !(rmin >= 0) || !(minimum_distance >= 0) || max_rounds < 1 ||
        !std::isfinite(lo) || !std::isfinite(hi) || !std::isfinite(rmax))
        return dem_set_error(ctx, DEM_E_INVALID, "bad generator ranges");
    if (n > 0 && (!x || !y || !z || !r)) return dem_set_error(ctx, DEM_E_INVALID, "null pointer");
    int rc = dem_check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (rc) return rc;
    if (rounds_out) *rounds_out = 0;
    if (n == 0) return DEM_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const double span = hi - lo;
    // workspace: inflated radii, two listed masks, pair buffer, counters
    double *rr = nullptr;
    int32_t *mask[2] = {nullptr, nullptr};
    int32_t *pairs = nullptr;
    int64_t *counts = nullptr;
    unsigned long long *listed = nullptr, listed_h = 0;
    int64_t counts_h[2] = {0, 0};
    int64_t cap = std::max<int64_t>(n, 1024);
    const int grid = std::max(1, std::min(ceil_div(n, 256), 8 * ctx->sm_count));
    auto cleanup = [&]() {
        cudaFree(rr);
        cudaFree(mask[0]);
        cudaFree(mask[1]);
        cudaFree(pairs);
        cudaFree(counts);
        cudaFree(listed);
    };
    rc = dem_check_cuda(ctx, cudaMalloc((void **)&rr, sizeof(double) * n), "generator workspace");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&mask[0], sizeof(int32_t) * n), "generator workspace");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&mask[1], sizeof(int32_t) * n), "generator workspace");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&pairs, sizeof(int32_t) * 2 * cap), "generator workspace");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&counts, sizeof(int64_t) * 2), "generator workspace");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&listed, sizeof(unsigned long long)), "generator workspace");
    if (rc) {
        cleanup();
        return rc;
    }
    const int table = next_pow2(2 * (int64_t)n);
    draw_radii_kernel<<<grid, 256, 0, counted(s)>>>(n, seed, rmin, rmax, 0.5 * minimum_distance, r, rr);
    int cur = 0;  // mask[cur]: droplets drawn this round (round 0: all)
    int round = 0;
    for (;; ++round) {
        if (round >= max_rounds) {
            cleanup();
            return dem_set_error(ctx, DEM_E_INVALID,
                                 "could not remove the overlaps in " + std::to_string(max_rounds) + " rounds");
        }
        const int32_t *drawn = round == 0 ? nullptr : mask[cur];
        draw_positions_kernel<<<grid, 256, 0, counted(s)>>>(n, seed, round, span, drawn, x, y, z);
        for (;;) {  // every overlapping pair; grow the buffer when it overflows
            rc = dem::launch_hash_detect(ctx, n, x, y, z, rr, span, periodic, table, pairs, cap, counts, s, periodic);
            if (!rc) rc = dem_check_cuda(ctx, cudaMemcpyAsync(counts_h, counts, sizeof(counts_h),
                                                              cudaMemcpyDeviceToHost, s), "generator count");
            if (!rc) rc = dem_check_cuda(ctx, cudaStreamSynchronize(s), "generator count");
            if (rc) {
                cleanup();
                return rc;
            }
            if (counts_h[0] <= cap) break;
            uint32_t flags = 0;  // clear the pair-overflow flag raised by the detection
            dem_device_errors(ctx, &flags, stream);
            cap = next_pow2(counts_h[0]);
            cudaFree(pairs);
            pairs = nullptr;
            rc = dem_check_cuda(ctx, cudaMalloc((void **)&pairs, sizeof(int32_t) * 2 * cap), "generator workspace");
            if (rc) {
                cleanup();
                return rc;
            }
        }
        if (counts_h[0] == 0) break;
        const int nxt = 1 - cur;
        rc = dem_check_cuda(ctx, cudaMemsetAsync(mask[nxt], 0, sizeof(int32_t) * n, s), "memset");
        if (!rc) rc = dem_check_cuda(ctx, cudaMemsetAsync(listed, 0, sizeof(unsigned long long), s), "memset");
        if (rc) {
            cleanup();
            return rc;
        }
        const int pgrid = std::max(1, std::min(ceil_div(counts_h[0], 256), 8 * ctx->sm_count));
        flag_overlaps_kernel<<<pgrid, 256, 0, counted(s)>>>(pairs, counts, drawn, mask[nxt], listed);
        rc = dem_check_cuda(ctx, cudaMemcpyAsync(&listed_h, listed, sizeof(listed_h), cudaMemcpyDeviceToHost, s),
                            "generator count");
        if (!rc) rc = dem_check_cuda(ctx, cudaStreamSynchronize(s), "generator count");
        if (rc) {
            cleanup();
            return rc;
        }
        cur = nxt;
        if (listed_h == 0) break;  // every overlap involves only droplets already accepted (cannot happen after round 0)
    }
    if (lo != 0.0) shift_kernel<<<grid, 256, 0, counted(s)>>>(n, lo, x, y, z);
    rc = dem_check_launch(ctx, "generator");
    if (!rc) rc = dem_check_cuda(ctx, cudaStreamSynchronize(s), "generator");
    cleanup();
    if (rounds_out) *rounds_out = round + 1;
    return rc;
}

}  // extern "C"
