// direct_vjp.cu -- adjoint (vector-Jacobian product) of the direct step velocity.
//
// The direct path moves droplet i with (euler_droplet_solver.py:121-125)
//   u_i = F_i / (gamma r_i) + V_i,
//   F_i = m r_i^3 sum_j r_j^3 f(d_ij),  d_ij = mic(x_j - x_i),  cut |d| > r_i + r_j
//         (direct_droplet_force_calculator.py:183-253),
//   V_i = eta sum_{j != i} G(e_ij) F_j,  e_ij = mic(x_i - x_j) = -d_ij,
//         G(e) = I / |e| + e e^T / |e|^3  (:354-411),
// with m = 12 pi eps0 eps_oil E^2.  Given a cotangent lambda on u this file
// computes lambda^T du/dx, lambda^T du/dr (collision cut and periodic wrap
// treated as non-differentiable); lambda^T du/dE = 2 lambda.u / E needs no kernel.
//
// Derivation used by the kernels:
//   * f(d) = P(d) / |d|^7 = grad(phi) / 3 with phi(d) = (|d|^2 - 3 dz^2) / |d|^5,
//     so df/dd = H(d) / 3 with H the (symmetric) Hessian of phi:
//       H = (-3 r^-5 + 15 dz^2 r^-7) I + (15 r^-7 - 105 dz^2 r^-9) d d^T
//           - 6 r^-5 z z^T + 30 dz r^-7 (z d^T + d z^T);
//   * the cotangent reaching the forces is
//       mu_i = lambda_i / (gamma r_i) + eta sum_{j != i} G(x_i - x_j) lambda_j
//     (G is even and symmetric: the Oseen pass applied to lambda);
//   * d(sum_k mu_k.F_k)/dx_i = (m/3) r_i^3 sum_j r_j^3 H(d_ij) (mu_j - mu_i),
//     d(sum_k mu_k.F_k)/dr_i = -3 m r_i^2 sum_j r_j^3 (mu_j - mu_i).f(d_ij);
//   * d(sum_k lambda_k.V_k)/dx_i = eta sum_{j != i} [K(e_ij; lambda_i, F_j) + K(e_ij; lambda_j, F_i)],
//       K(e; a, b) = grad_e(a^T G(e) b) = [(e.b) a + (e.a) b - (a.b) e] / |e|^3 - 3 (a.e)(e.b) e / |e|^5;
//   * d(lambda_i.F_i / (gamma r_i))/dr_i = -lambda_i.F_i / (gamma r_i^2).
// Everything is FP64.  Both O(N^2) passes (mu and the pair terms) cut the j range
// into chunks, one CTA per (128 droplets i, chunk): at N = 16,384 one thread per i
// alone would fill 128 CTAs on 148 SMs.  The chunks' partial sums are added in
// chunk order (deterministic).  1 / |d| comes from an FP32 estimate refined by
// two Newton steps in FP64 (rsqrt_nr), not from an IEEE square root and division.
#include "common.cuh"

namespace dem {

constexpr int VJP_THREADS = 128;
constexpr int VJP_TILE = 128;

// 1 / sqrt(x) for x > 0 by Newton's method on f(y) = y^-2 - x: y <- y (3 - x y^2) / 2,
// which converges quadratically, from the FP32 estimate rsqrtf (relative error
// ~2^-23): two steps reach FP64 rounding.  Outside FP32's range: sqrt and a division.
__device__ __forceinline__ double rsqrt_nr(double x) {
    if (!(x > 1e-30 && x < 1e30)) return 1.0 / sqrt(x);
    double y = (double)rsqrtf((float)x);
    const double hx = 0.5 * x;
    y = y * fma(-hx, y * y, 1.5);
    y = y * fma(-hx, y * y, 1.5);
    return y;
}

// The j range [j0, j1) of split blockIdx.y.
struct VjpSplit {
    int chunk;  // j per split (a multiple of VJP_TILE)
    int splits;
};

// Oseen pass applied to lambda, partial sums of split s: part[(3 s + c) n + i] = sum_j G(e_ij) lambda_j
// over the split's j != i (e = mic(x_i - x_j), G(e) = I / |e| + e e^T / |e|^3).
template <bool PER>
__global__ void __launch_bounds__(VJP_THREADS) vjp_oseen_kernel(int n, const double *__restrict__ x,
                                                                const double *__restrict__ y,
                                                                const double *__restrict__ z,
                                                                const double *__restrict__ lx,
                                                                const double *__restrict__ ly,
                                                                const double *__restrict__ lz, double L, double halfL,
                                                                VjpSplit sp, double *__restrict__ part) {
    __shared__ double sx[VJP_TILE], sy[VJP_TILE], sz[VJP_TILE], slx[VJP_TILE], sly[VJP_TILE], slz[VJP_TILE];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    const double xi = active ? x[i] : 0.0, yi = active ? y[i] : 0.0, zi = active ? z[i] : 0.0;
    const int j0 = blockIdx.y * sp.chunk, j1 = min(n, j0 + sp.chunk);
    double ux = 0.0, uy = 0.0, uz = 0.0;
    for (int t0 = j0; t0 < j1; t0 += VJP_TILE) {
        __syncthreads();
        for (int k = threadIdx.x; k < VJP_TILE; k += blockDim.x) {
            const int j = t0 + k;
            if (j < j1) {
                sx[k] = x[j];
                sy[k] = y[j];
                sz[k] = z[j];
                slx[k] = lx[j];
                sly[k] = ly[j];
                slz[k] = lz[j];
            }
        }
        __syncthreads();
        const int cnt = min(VJP_TILE, j1 - t0);
        if (!active) continue;
        for (int k = 0; k < cnt; ++k) {
            if (t0 + k == i) continue;
            double ex = xi - sx[k], ey = yi - sy[k], ez = zi - sz[k];
            if (PER) {
                ex = mic64(ex, L, halfL);
                ey = mic64(ey, L, halfL);
                ez = mic64(ez, L, halfL);
            }
            const double r2 = ex * ex + ey * ey + ez * ez;
            const double ir = rsqrt_nr(r2), ir2 = ir * ir;
            const double el = (ex * slx[k] + ey * sly[k] + ez * slz[k]) * ir2;
            ux += (slx[k] + ex * el) * ir;
            uy += (sly[k] + ey * el) * ir;
            uz += (slz[k] + ez * el) * ir;
        }
    }
    if (!active) return;
    double *o = part + (size_t)blockIdx.y * 3 * n;
    o[i] = ux;
    o[n + i] = uy;
    o[2 * (size_t)n + i] = uz;
}

// mu_i = eta sum_s part_s + lambda_i / (gamma r_i)  (splits in order)
__global__ void vjp_mu_kernel(int n, int splits, const double *__restrict__ part, const double *__restrict__ r,
                              const double *__restrict__ lx, const double *__restrict__ ly,
                              const double *__restrict__ lz, double eta, double stokes, double *__restrict__ mx,
                              double *__restrict__ my, double *__restrict__ mz) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ux = 0.0, uy = 0.0, uz = 0.0;
        for (int s = 0; s < splits; ++s) {
            const double *o = part + (size_t)s * 3 * n;
            ux += o[i];
            uy += o[n + i];
            uz += o[2 * (size_t)n + i];
        }
        const double a = 1.0 / (stokes * r[i]);
        mx[i] = eta * ux + a * lx[i];
        my[i] = eta * uy + a * ly[i];
        mz[i] = eta * uz + a * lz[i];
    }
}

struct VjpArgs {
    int n;
    const double *x, *y, *z, *r;
    const double *fx, *fy, *fz;  // forces at this state
    const double *lx, *ly, *lz;  // lambda: cotangent on u
    const double *mx, *my, *mz;  // mu: cotangent on F
    double m_const, eta, stokes, L, halfL;
    double *gx, *gy, *gz, *gr;
    VjpSplit sp;
    double *part;  // [splits][7][n] partial sums (vjp_pair_kernel)
};

// Partial sums of split s over its j != i:
//   part[(7 s + 0..2) n + i] = sum_j r_j^3 H(d_ij) (mu_j - mu_i)   (force terms, cut |d| > r_i + r_j)
//   part[(7 s + 3) n + i]    = sum_j r_j^3 (mu_j - mu_i).f(d_ij)
//   part[(7 s + 4..6) n + i] = sum_j K(e_ij; lambda_i, F_j) + K(e_ij; lambda_j, F_i)
template <bool PER>
__global__ void __launch_bounds__(VJP_THREADS) vjp_pair_kernel(const VjpArgs a) {
    __shared__ double sx[VJP_TILE], sy[VJP_TILE], sz[VJP_TILE], sr[VJP_TILE];
    __shared__ double smx[VJP_TILE], smy[VJP_TILE], smz[VJP_TILE];
    __shared__ double slx[VJP_TILE], sly[VJP_TILE], slz[VJP_TILE];
    __shared__ double sfx[VJP_TILE], sfy[VJP_TILE], sfz[VJP_TILE];
    const int n = a.n;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    double xi = 0, yi = 0, zi = 0, ri = 0, mix = 0, miy = 0, miz = 0, lix = 0, liy = 0, liz = 0, fix = 0, fiy = 0,
           fiz = 0;
    if (active) {
        xi = a.x[i];
        yi = a.y[i];
        zi = a.z[i];
        ri = a.r[i];
        mix = a.mx[i];
        miy = a.my[i];
        miz = a.mz[i];
        lix = a.lx[i];
        liy = a.ly[i];
        liz = a.lz[i];
        fix = a.fx[i];
        fiy = a.fy[i];
        fiz = a.fz[i];
    }
    double hx = 0, hy = 0, hz = 0;  // sum_j r_j^3 H (mu_j - mu_i)
    double gR = 0;                  // sum_j r_j^3 (mu_j - mu_i).f
    double kx = 0, ky = 0, kz = 0;  // sum_j K(e; lambda_i, F_j) + K(e; lambda_j, F_i)
    const int j0 = blockIdx.y * a.sp.chunk, j1 = min(n, j0 + a.sp.chunk);
    for (int t0 = j0; t0 < j1; t0 += VJP_TILE) {
        __syncthreads();
        for (int k = threadIdx.x; k < VJP_TILE; k += blockDim.x) {
            const int j = t0 + k;
            if (j < j1) {
                sx[k] = a.x[j];
                sy[k] = a.y[j];
                sz[k] = a.z[j];
                sr[k] = a.r[j];
                smx[k] = a.mx[j];
                smy[k] = a.my[j];
                smz[k] = a.mz[j];
                slx[k] = a.lx[j];
                sly[k] = a.ly[j];
                slz[k] = a.lz[j];
                sfx[k] = a.fx[j];
                sfy[k] = a.fy[j];
                sfz[k] = a.fz[j];
            }
        }
        __syncthreads();
        const int cnt = min(VJP_TILE, j1 - t0);
        if (!active) continue;
        for (int k = 0; k < cnt; ++k) {
            if (t0 + k == i) continue;
            double dx = sx[k] - xi, dy = sy[k] - yi, dz = sz[k] - zi;  // d = x_j - x_i
            if (PER) {
                dx = mic64(dx, a.L, a.halfL);
                dy = mic64(dy, a.L, a.halfL);
                dz = mic64(dz, a.L, a.halfL);
            }
            const double r2 = dx * dx + dy * dy + dz * dz;
            const double ir = rsqrt_nr(r2), ir2 = ir * ir, ir3 = ir2 * ir, ir5 = ir3 * ir2;
            if (r2 * ir > ri + sr[k]) {  // force terms (contact cut of the forward pass, |d| = r2 / |d|)
                const double ir7 = ir5 * ir2, ir9 = ir7 * ir2;
                const double w = ipow3(sr[k]);
                const double nx = smx[k] - mix, ny = smy[k] - miy, nz = smz[k] - miz;
                const double dn = dx * nx + dy * ny + dz * nz;
                const double z2 = dz * dz;
                const double c1 = -3.0 * ir5 + 15.0 * z2 * ir7;
                const double c2 = (15.0 * ir7 - 105.0 * z2 * ir9) * dn;
                const double c3 = 30.0 * dz * ir7 * nz;
                hx += w * (c1 * nx + c2 * dx + c3 * dx);
                hy += w * (c1 * ny + c2 * dy + c3 * dy);
                hz += w * (c1 * nz + c2 * dz - 6.0 * ir5 * nz + 30.0 * dz * ir7 * dn + c3 * dz);
                const double axy = (4.0 * z2 - dx * dx - dy * dy) * ir7;
                const double az = (2.0 * z2 - 3.0 * dx * dx - 3.0 * dy * dy) * ir7;
                gR += w * (nx * dx * axy + ny * dy * axy + nz * dz * az);
            }
            // Oseen terms with e = x_i - x_j = -d (no cut)
            const double ex = -dx, ey = -dy, ez = -dz;
            {  // K(e; lambda_i, F_j)
                const double ax_ = lix, ay_ = liy, az_ = liz, bx = sfx[k], by = sfy[k], bz = sfz[k];
                const double eb = ex * bx + ey * by + ez * bz, ea = ex * ax_ + ey * ay_ + ez * az_;
                const double ab = ax_ * bx + ay_ * by + az_ * bz;
                const double q = 3.0 * ea * eb * ir5;
                kx += (eb * ax_ + ea * bx - ab * ex) * ir3 - q * ex;
                ky += (eb * ay_ + ea * by - ab * ey) * ir3 - q * ey;
                kz += (eb * az_ + ea * bz - ab * ez) * ir3 - q * ez;
            }
            {  // K(e; lambda_j, F_i)
                const double ax_ = slx[k], ay_ = sly[k], az_ = slz[k], bx = fix, by = fiy, bz = fiz;
                const double eb = ex * bx + ey * by + ez * bz, ea = ex * ax_ + ey * ay_ + ez * az_;
                const double ab = ax_ * bx + ay_ * by + az_ * bz;
                const double q = 3.0 * ea * eb * ir5;
                kx += (eb * ax_ + ea * bx - ab * ex) * ir3 - q * ex;
                ky += (eb * ay_ + ea * by - ab * ey) * ir3 - q * ey;
                kz += (eb * az_ + ea * bz - ab * ez) * ir3 - q * ez;
            }
        }
    }
    if (!active) return;
    double *o = a.part + (size_t)blockIdx.y * 7 * n;
    o[i] = hx;
    o[n + i] = hy;
    o[2 * (size_t)n + i] = hz;
    o[3 * (size_t)n + i] = gR;
    o[4 * (size_t)n + i] = kx;
    o[5 * (size_t)n + i] = ky;
    o[6 * (size_t)n + i] = kz;
}

// The gradients from the splits' partial sums (in split order).
__global__ void vjp_finish_kernel(const VjpArgs a) {
    const int n = a.n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int s = 0; s < a.sp.splits; ++s) {
            const double *o = a.part + (size_t)s * 7 * n;
#pragma unroll
            for (int c = 0; c < 7; ++c) v[c] += o[(size_t)c * n + i];
        }
        const double ri = a.r[i];
        const double cf = a.m_const / 3.0 * ipow3(ri);
        a.gx[i] = cf * v[0] + a.eta * v[4];
        a.gy[i] = cf * v[1] + a.eta * v[5];
        a.gz[i] = cf * v[2] + a.eta * v[6];
        const double lf = a.lx[i] * a.fx[i] + a.ly[i] * a.fy[i] + a.lz[i] * a.fz[i];
        a.gr[i] = -3.0 * a.m_const * ri * ri * v[3] - lf / (a.stokes * ri * ri);
    }
}

// j chunks such that the (i block, chunk) grid holds >= 8 CTAs per SM
static VjpSplit vjp_split(const dem_ctx *ctx, int n) {
    const int iblocks = ceil_div(n, VJP_THREADS);
    const int want = max(1, ceil_div(8 * ctx->sm_count, iblocks));
    int chunk = ceil_div(ceil_div(n, want), VJP_TILE) * VJP_TILE;
    if (chunk < VJP_TILE) chunk = VJP_TILE;
    VjpSplit sp;
    sp.chunk = chunk;
    sp.splits = max(1, ceil_div(n, chunk));
    return sp;
}

int launch_direct_vjp(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                      const double *fx, const double *fy, const double *fz, const double *lx, const double *ly,
                      const double *lz, double m_const, double eta, double stokes, double L, int periodic,
                      double *mx, double *my, double *mz, double *gx, double *gy, double *gz, double *gr,
                      cudaStream_t s) {
    if (n == 0) return DEM_OK;
    const VjpSplit sp = vjp_split(ctx, n);
    // partial sums: [splits][7][n] doubles in the context's [splits][3][capacity] array
    int rc = dem_ensure_partials(ctx, ceil_div(7 * sp.splits, 3));
    if (rc) return rc;
    double *part = ctx->partial;
    const dim3 grid(ceil_div(n, VJP_THREADS), sp.splits);
    const int egrid = min(ceil_div(n, 256), 8 * ctx->sm_count);
    // mu = eta (Oseen pass applied to lambda) + lambda / (gamma r)
    if (periodic)
        vjp_oseen_kernel<true><<<grid, VJP_THREADS, 0, counted(s)>>>(n, x, y, z, lx, ly, lz, L, 0.5 * L, sp, part);
    else
        vjp_oseen_kernel<false><<<grid, VJP_THREADS, 0, counted(s)>>>(n, x, y, z, lx, ly, lz, L, 0.5 * L, sp, part);
    vjp_mu_kernel<<<egrid, 256, 0, counted(s)>>>(n, sp.splits, part, r, lx, ly, lz, eta, stokes, mx, my, mz);
    if ((rc = dem_check_launch(ctx, "vjp mu"))) return rc;
    VjpArgs a{n, x, y, z, r, fx, fy, fz, lx, ly, lz, mx, my, mz, m_const, eta, stokes, L, 0.5 * L, gx, gy, gz, gr,
              sp, part};
    dem_prof_begin(ctx, "vjp_pass", s);
    if (periodic)
        vjp_pair_kernel<true><<<grid, VJP_THREADS, 0, counted(s)>>>(a);
    else
        vjp_pair_kernel<false><<<grid, VJP_THREADS, 0, counted(s)>>>(a);
    vjp_finish_kernel<<<egrid, 256, 0, counted(s)>>>(a);
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "vjp pair pass");
}

}  // namespace dem
