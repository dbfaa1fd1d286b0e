// direct_fp64.cu -- plain-FP64 direct O(N^2) passes (the reference drop-in).
//
// One thread owns one droplet i and sums its pair terms over j = 0..n-1 in
// ascending order, exactly like the reference's serial inner loop, with every
// expression evaluated in the reference's order.  This file is compiled with
// -fmad=false so no multiply-add is contracted: each operation rounds once,
// and the results are bit-identical to the CPU restatement of
//   dem/force_calculator/direct_droplet_force_calculator.py:183-253 (forces)
//   dem/force_calculator/direct_droplet_force_calculator.py:354-411 (convection).
//
// j-tiles (x, y, z, r, r^3) are staged in shared memory and read as
// broadcasts; the pair work is FP64-pipe bound (IEEE sqrt / division).
//
// With the periodic-image correction loaded, the convection kernel adds each
// pair's correction term right after its Stokeslet term and the self term
// after the loop (:413-464), bit-identical to the CPU restatement.
#include "common.cuh"
#include "corr.cuh"

namespace dem {

constexpr int F64_THREADS = 128;
constexpr int F64_TILE = 128;

template <bool PERIODIC>
__global__ void __launch_bounds__(F64_THREADS) direct_force_fp64_kernel(int n, const double *__restrict__ x,
                                                                        const double *__restrict__ y,
                                                                        const double *__restrict__ z,
                                                                        const double *__restrict__ r, double m_const,
                                                                        double L, double halfL, double *__restrict__ fx,
                                                                        double *__restrict__ fy, double *__restrict__ fz) {
    __shared__ double sx[F64_TILE], sy[F64_TILE], sz[F64_TILE], sr[F64_TILE], sr3[F64_TILE];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    double xi = 0, yi = 0, zi = 0, ri = 0, mri3 = 0;
    if (active) {
        xi = x[i];
        yi = y[i];
        zi = z[i];
        ri = r[i];
        mri3 = m_const * ipow3(ri);  // (m_const * r_i**3) is the first product of :189
    }
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    for (int t0 = 0; t0 < n; t0 += F64_TILE) {
        __syncthreads();
        for (int k = threadIdx.x; k < F64_TILE; k += blockDim.x) {
            const int j = t0 + k;
            if (j < n) {
                sx[k] = x[j];
                sy[k] = y[j];
                sz[k] = z[j];
                const double rj = r[j];
                sr[k] = rj;
                sr3[k] = ipow3(rj);
            }
        }
        __syncthreads();
        const int cnt = min(F64_TILE, n - t0);
        if (!active) continue;
        for (int k = 0; k < cnt; ++k) {
            if (t0 + k == i) continue;
            double dx = sx[k] - xi, dy = sy[k] - yi, dz = sz[k] - zi;
            if (PERIODIC) {
                dx = mic64(dx, L, halfL);
                dy = mic64(dy, L, halfL);
                dz = mic64(dz, L, halfL);
            }
            const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
            const double r_mag = sqrt(dx2 + dy2 + dz2);
            if (r_mag > ri + sr[k]) {
                const double M = mri3 * sr3[k] / ipow7(r_mag);
                const double fxy = M * (4 * dz2 - dx2 - dy2);
                Fx += fxy * dx;
                Fy += fxy * dy;
                Fz += M * (2 * dz2 - 3 * dx2 - 3 * dy2) * dz;
            }
        }
    }
    if (active) {
        fx[i] = Fx;
        fy[i] = Fy;
        fz[i] = Fz;
    }
}

template <bool PERIODIC, bool CORR>
__global__ void __launch_bounds__(F64_THREADS) direct_convection_fp64_kernel(
    int n, const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z,
    const double *__restrict__ fx, const double *__restrict__ fy, const double *__restrict__ fz, double eta,
    double L, double halfL, CorrDev corr, double *__restrict__ vx, double *__restrict__ vy,
    double *__restrict__ vz) {
    __shared__ double sx[F64_TILE], sy[F64_TILE], sz[F64_TILE], sfx[F64_TILE], sfy[F64_TILE], sfz[F64_TILE];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    double xi = 0, yi = 0, zi = 0;
    if (active) {
        xi = x[i];
        yi = y[i];
        zi = z[i];
    }
    double Cx = 0.0, Cy = 0.0, Cz = 0.0;
    for (int t0 = 0; t0 < n; t0 += F64_TILE) {
        __syncthreads();
        for (int k = threadIdx.x; k < F64_TILE; k += blockDim.x) {
            const int j = t0 + k;
            if (j < n) {
                sx[k] = x[j];
                sy[k] = y[j];
                sz[k] = z[j];
                sfx[k] = fx[j];
                sfy[k] = fy[j];
                sfz[k] = fz[j];
            }
        }
        __syncthreads();
        const int cnt = min(F64_TILE, n - t0);
        if (!active) continue;
        for (int k = 0; k < cnt; ++k) {
            if (t0 + k == i) continue;
            double X = xi - sx[k], Y = yi - sy[k], Z = zi - sz[k];
            if (PERIODIC) {
                X = mic64(X, L, halfL);
                Y = mic64(Y, L, halfL);
                Z = mic64(Z, L, halfL);
            }
            const double rr = sqrt(X * X + Y * Y + Z * Z);
            const double r3 = ipow3(rr);
            const double Fx = sfx[k], Fy = sfy[k], Fz = sfz[k];
            const double inv_r = 1 / rr;
            const double xy = (X * Y) / r3, xz = (X * Z) / r3, yz = (Y * Z) / r3;
            Cx += eta * ((inv_r + (X * X) / r3) * Fx + xy * Fy + xz * Fz);
            Cy += eta * (xy * Fx + (inv_r + (Y * Y) / r3) * Fy + yz * Fz);
            Cz += eta * (xz * Fx + yz * Fy + (inv_r + (Z * Z) / r3) * Fz);
            if (CORR) corr_pair64(corr, X, Y, Z, Fx, Fy, Fz, Cx, Cy, Cz);
        }
    }
    if (CORR && active) {
        Cx += corr.g_self * fx[i];
        Cy += corr.g_self * fy[i];
        Cz += corr.g_self * fz[i];
    }
    if (active) {
        vx[i] = Cx;
        vy[i] = Cy;
        vz[i] = Cz;
    }
}

int launch_direct_forces_fp64(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                              const double *r, double m_const, double L, int periodic, double *fx, double *fy,
                              double *fz, cudaStream_t s) {
    const int grid = ceil_div(n, F64_THREADS);
    dem_prof_begin(ctx, "fp64_force_pass", s);
    if (periodic)
        direct_force_fp64_kernel<true><<<grid, F64_THREADS, 0, counted(s)>>>(n, x, y, z, r, m_const, L, L * 0.5, fx, fy, fz);
    else
        direct_force_fp64_kernel<false><<<grid, F64_THREADS, 0, counted(s)>>>(n, x, y, z, r, m_const, L, L * 0.5, fx, fy, fz);
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "direct_force_fp64");
}

int launch_direct_convection_fp64(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                                  const double *fx, const double *fy, const double *fz, double eta, double L,
                                  int periodic, double *vx, double *vy, double *vz, cudaStream_t s) {
    const int grid = ceil_div(n, F64_THREADS);
    dem_prof_begin(ctx, "fp64_convection_pass", s);
    const CorrDev none{};
    if (periodic)
        direct_convection_fp64_kernel<true, false>
            <<<grid, F64_THREADS, 0, counted(s)>>>(n, x, y, z, fx, fy, fz, eta, L, L * 0.5, none, vx, vy, vz);
    else
        direct_convection_fp64_kernel<false, false>
            <<<grid, F64_THREADS, 0, counted(s)>>>(n, x, y, z, fx, fy, fz, eta, L, L * 0.5, none, vx, vy, vz);
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "direct_convection_fp64");
}

int launch_direct_convection_fp64_corr(dem_ctx *ctx, const dem_corr *c, int n, const double *x, const double *y,
                                       const double *z, const double *fx, const double *fy, const double *fz,
                                       double eta, double L, int periodic, double *vx, double *vy, double *vz,
                                       cudaStream_t s) {
    const int grid = ceil_div(n, F64_THREADS);
    const CorrDev cv = corr_view(c);
    dem_prof_begin(ctx, "fp64_convection_corr_pass", s);
    if (periodic)
        direct_convection_fp64_kernel<true, true>
            <<<grid, F64_THREADS, 0, counted(s)>>>(n, x, y, z, fx, fy, fz, eta, L, L * 0.5, cv, vx, vy, vz);
    else
        direct_convection_fp64_kernel<false, true>
            <<<grid, F64_THREADS, 0, counted(s)>>>(n, x, y, z, fx, fy, fz, eta, L, L * 0.5, cv, vx, vy, vz);
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "direct_convection_fp64_corr");
}

}  // namespace dem
