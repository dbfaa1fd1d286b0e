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
// Everything is FP64; one thread per droplet i, j tiles staged in shared memory.
#include "common.cuh"

namespace dem {

int launch_direct_convection_fp64(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                                  const double *fx, const double *fy, const double *fz, double eta, double L,
                                  int periodic, double *vx, double *vy, double *vz, cudaStream_t s);

constexpr int VJP_THREADS = 128;
constexpr int VJP_TILE = 128;

// mu_i += lambda_i / (gamma r_i)
__global__ void vjp_mu_kernel(int n, const double *__restrict__ r, const double *__restrict__ lx,
                              const double *__restrict__ ly, const double *__restrict__ lz, double stokes,
                              double *__restrict__ mx, double *__restrict__ my, double *__restrict__ mz) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double a = 1.0 / (stokes * r[i]);
        mx[i] += a * lx[i];
        my[i] += a * ly[i];
        mz[i] += a * lz[i];
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
};

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
    for (int t0 = 0; t0 < n; t0 += VJP_TILE) {
        __syncthreads();
        for (int k = threadIdx.x; k < VJP_TILE; k += blockDim.x) {
            const int j = t0 + k;
            if (j < n) {
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
        const int cnt = min(VJP_TILE, n - t0);
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
            const double rr = sqrt(r2);
            const double ir = 1.0 / rr, ir2 = ir * ir, ir3 = ir2 * ir, ir5 = ir3 * ir2;
            if (rr > ri + sr[k]) {  // force terms (contact cut of the forward pass)
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
    const double ri3 = ipow3(ri);
    const double cf = a.m_const / 3.0 * ri3;
    a.gx[i] = cf * hx + a.eta * kx;
    a.gy[i] = cf * hy + a.eta * ky;
    a.gz[i] = cf * hz + a.eta * kz;
    const double lf = lix * fix + liy * fiy + liz * fiz;
    a.gr[i] = -3.0 * a.m_const * ri * ri * gR - lf / (a.stokes * ri * ri);
}

int launch_direct_vjp(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                      const double *fx, const double *fy, const double *fz, const double *lx, const double *ly,
                      const double *lz, double m_const, double eta, double stokes, double L, int periodic,
                      double *mx, double *my, double *mz, double *gx, double *gy, double *gz, double *gr,
                      cudaStream_t s) {
    if (n == 0) return DEM_OK;
    // mu = Oseen pass applied to lambda, plus lambda / (gamma r)
    int rc = launch_direct_convection_fp64(ctx, n, x, y, z, lx, ly, lz, eta, L, periodic, mx, my, mz, s);
    if (rc) return rc;
    const int egrid = min(ceil_div(n, 256), 8 * ctx->sm_count);
    vjp_mu_kernel<<<egrid, 256, 0, counted(s)>>>(n, r, lx, ly, lz, stokes, mx, my, mz);
    if ((rc = dem_check_launch(ctx, "vjp mu"))) return rc;
    VjpArgs a{n, x, y, z, r, fx, fy, fz, lx, ly, lz, mx, my, mz, m_const, eta, stokes, L, 0.5 * L, gx, gy, gz, gr};
    const int grid = ceil_div(n, VJP_THREADS);
    dem_prof_begin(ctx, "vjp_pass", s);
    if (periodic)
        vjp_pair_kernel<true><<<grid, VJP_THREADS, 0, counted(s)>>>(a);
    else
        vjp_pair_kernel<false><<<grid, VJP_THREADS, 0, counted(s)>>>(a);
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "vjp pair pass");
}

}  // namespace dem
