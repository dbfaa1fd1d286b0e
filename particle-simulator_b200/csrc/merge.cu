// merge.cu -- coalescence of colliding droplets on the device.
//
// DropletSolution.generate_next_solution, dem/solution/droplet_solution.py:208-287:
//   * pairs are visited in (i, j) order; a pair is skipped when either droplet
//     has already merged (greedy, lowest index first);
//   * r_new = (r_a**3 + r_b**3) ** (1/3),
//     x_new = (x_a r_a**3 + x_b r_b**3) / (r_a**3 + r_b**3)   (no minimum image);
//   * the merged droplets are deleted (order of the survivors kept) and the new
//     ones appended at the end in merge order.
// numpy evaluates r**3 and v**(1/3) with libm pow, which rounds (all but
// never-seen cases) correctly; this file computes both correctly rounded from
// exact error-free products (Dekker/FMA two-product), Newton's correction of
// the cube root and a first-order correction for the exponent RN(1/3), which
// is 1/3 - 2^-54/3.  Compiled with -fmad=false (no implicit contraction).
#include "common.cuh"
#include "scan.cuh"

namespace dem {

// RN(r^3): r*r = p + e exactly, r^3 = r*p + r*e; one rounding of the sum.
__device__ __forceinline__ double cube_rn(double r) {
    const double p = r * r;
    const double e = fma(r, r, -p);
    return fma(r, p, r * e);
}

// RN(v ** RN(1/3)) for normal positive finite v.
__device__ __forceinline__ double pow_third_rn(double v) {
    if (!(v > 1e-290) || !isfinite(v)) return pow(v, 1.0 / 3.0);
    const double c0 = cbrt(v);
    const double ph = c0 * c0;
    const double pl = fma(c0, c0, -ph);
    const double qh = c0 * ph;
    const double ql = fma(c0, ph, -qh);
    const double res = ((v - qh) - ql) - c0 * pl;  // v - c0^3
    const double corr = res / (3.0 * ph);           // Newton step of the cube root
    // v^(1/3 - d) = cbrt(v) * (1 - d ln v + O(d^2)),  d = 2^-54 / 3
    const double kappa = -(0x1p-54 / 3.0) * log(v);
    return c0 + (corr + c0 * kappa);
}

// Greedy selection: one thread walks the pairs in order (the only serial part).
__global__ void merge_select_kernel(int n, const int32_t *__restrict__ pairs, const int64_t *__restrict__ num_pairs,
                                    int32_t *__restrict__ consumed, int32_t *__restrict__ sel,
                                    int32_t *__restrict__ m_out, uint32_t *err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int64_t k = *num_pairs;
    int32_t m = 0;
    for (int64_t p = 0; p < k; ++p) {
        const int32_t a = pairs[2 * p], b = pairs[2 * p + 1];
        if (a < 0 || b < 0 || a >= n || b >= n || a == b) {
            raise_device_error(err, DEM_DEVERR_PAIR_OVERFLOW);
            continue;
        }
        if (consumed[a] || consumed[b]) continue;
        consumed[a] = 1;
        consumed[b] = 1;
        sel[2 * m] = a;
        sel[2 * m + 1] = b;
        ++m;
    }
    *m_out = m;
}

__global__ void merge_compute_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                     const double *__restrict__ z, const double *__restrict__ r,
                                     const int32_t *__restrict__ sel, const int32_t *__restrict__ m_in,
                                     double *__restrict__ merged) {
    const int32_t m = *m_in;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int32_t a = sel[2 * q], b = sel[2 * q + 1];
        const double c1 = cube_rn(r[a]), c2 = cube_rn(r[b]);
        const double v = c1 + c2;
        merged[4 * q + 0] = (x[a] * c1 + x[b] * c2) / v;
        merged[4 * q + 1] = (y[a] * c1 + y[b] * c2) / v;
        merged[4 * q + 2] = (z[a] * c1 + z[b] * c2) / v;
        merged[4 * q + 3] = pow_third_rn(v);
    }
}

__global__ void merge_compact_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                     const double *__restrict__ z, const double *__restrict__ r,
                                     const int32_t *__restrict__ consumed, const int32_t *__restrict__ consumed_before,
                                     const double *__restrict__ merged, const int32_t *__restrict__ sel,
                                     const int32_t *__restrict__ m_in, double *__restrict__ xo, double *__restrict__ yo,
                                     double *__restrict__ zo, double *__restrict__ ro, int32_t *__restrict__ n_out,
                                     int32_t *__restrict__ merged_pairs) {
    const int32_t m = *m_in;
    const int32_t survivors = n - 2 * m;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!consumed[i]) {
            const int32_t w = i - consumed_before[i];
            xo[w] = x[i];
            yo[w] = y[i];
            zo[w] = z[i];
            ro[w] = r[i];
        }
        if (i < m) {
            const int32_t w = survivors + i;
            xo[w] = merged[4 * i + 0];
            yo[w] = merged[4 * i + 1];
            zo[w] = merged[4 * i + 2];
            ro[w] = merged[4 * i + 3];
            if (merged_pairs) {
                merged_pairs[2 * i] = sel[2 * i];
                merged_pairs[2 * i + 1] = sel[2 * i + 1];
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = n - m;
}

int launch_merge(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                 const int32_t *pairs, const int64_t *num_pairs, double *xo, double *yo, double *zo, double *ro,
                 int32_t *n_out, int32_t *merged_pairs, cudaStream_t s) {
    int rc = dem_check_cuda(ctx, cudaMemsetAsync(ctx->flags, 0, sizeof(int32_t) * (size_t)(n + 1), s), "memset");
    if (rc) return rc;
    // The selection list holds at most n/2 pairs (2 * (n / 2) int32); it lives in
    // the hash detector's per-droplet offset buffer (int64[capacity + 1]), which
    // is free once the pairs have been written.
    int32_t *sel = reinterpret_cast<int32_t *>(ctx->pair_offset);
    merge_select_kernel<<<1, 32, 0, counted(s)>>>(n, pairs, num_pairs, ctx->flags, sel, ctx->merged_cnt, ctx->d_err);
    const int grid = max(1, min(ceil_div(n, 256), 8 * ctx->sm_count));
    merge_compute_kernel<<<grid, 256, 0, counted(s)>>>(x, y, z, r, sel, ctx->merged_cnt, ctx->merged_buf);
    rc = dem_check_launch(ctx, "merge select");
    if (rc) return rc;
    rc = exclusive_scan<int32_t, int32_t>(ctx, ctx->flags, ctx->keep_off, n, s);
    if (rc) return rc;
    merge_compact_kernel<<<grid, 256, 0, counted(s)>>>(n, x, y, z, r, ctx->flags, ctx->keep_off, ctx->merged_buf, sel,
                                              ctx->merged_cnt, xo, yo, zo, ro, n_out, merged_pairs);
    return dem_check_launch(ctx, "merge compact");
}

}  // namespace dem
