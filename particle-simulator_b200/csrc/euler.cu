// euler.cu -- explicit Euler update with the periodic wrap.
//
// Direct path, dem/solver/euler_droplet_solver.py:121-131:
//   v_mig = F / (stokes_factor * r);  x += (v_mig + v_conv) * dt;  x %= L
// Tree path, :119 and :130-131:  x += v_total * dt;  x %= L
// `%=` is numpy's float remainder (fmod, then + L for a negative result).
// Compiled with -fmad=false: each operation rounds once, as in numpy.
#include "common.cuh"

namespace dem {

__global__ void euler_direct_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                    const double *__restrict__ z, const double *__restrict__ r,
                                    const double *__restrict__ fx, const double *__restrict__ fy,
                                    const double *__restrict__ fz, const double *__restrict__ vx,
                                    const double *__restrict__ vy, const double *__restrict__ vz, double stokes,
                                    double dt, double L, int periodic, double *xo, double *yo, double *zo) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double denom = stokes * r[i];
        double px = x[i] + (fx[i] / denom + vx[i]) * dt;
        double py = y[i] + (fy[i] / denom + vy[i]) * dt;
        double pz = z[i] + (fz[i] / denom + vz[i]) * dt;
        if (periodic) {
            px = np_remainder(px, L);
            py = np_remainder(py, L);
            pz = np_remainder(pz, L);
        }
        xo[i] = px;
        yo[i] = py;
        zo[i] = pz;
    }
}

__global__ void euler_total_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                   const double *__restrict__ z, const double *__restrict__ vx,
                                   const double *__restrict__ vy, const double *__restrict__ vz, double dt, double L,
                                   int periodic, double *xo, double *yo, double *zo) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double px = x[i] + vx[i] * dt, py = y[i] + vy[i] * dt, pz = z[i] + vz[i] * dt;
        if (periodic) {
            px = np_remainder(px, L);
            py = np_remainder(py, L);
            pz = np_remainder(pz, L);
        }
        xo[i] = px;
        yo[i] = py;
        zo[i] = pz;
    }
}

// Several independent boxes: droplets [off[b], off[b+1]) live in a box of side L[b].
__global__ void euler_direct_boxes_kernel(int n, int nbox, const int *__restrict__ off, const double *__restrict__ Lb,
                                          const double *__restrict__ x, const double *__restrict__ y,
                                          const double *__restrict__ z, const double *__restrict__ r,
                                          const double *__restrict__ fx, const double *__restrict__ fy,
                                          const double *__restrict__ fz, const double *__restrict__ vx,
                                          const double *__restrict__ vy, const double *__restrict__ vz, double stokes,
                                          double dt, int periodic, double *xo, double *yo, double *zo) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int lo = 0, hi = nbox - 1;  // box of droplet i: the last b with off[b] <= i
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (off[mid] <= i)
                lo = mid;
            else
                hi = mid - 1;
        }
        const double L = Lb[lo];
        const double denom = stokes * r[i];
        double px = x[i] + (fx[i] / denom + vx[i]) * dt;
        double py = y[i] + (fy[i] / denom + vy[i]) * dt;
        double pz = z[i] + (fz[i] / denom + vz[i]) * dt;
        if (periodic) {
            px = np_remainder(px, L);
            py = np_remainder(py, L);
            pz = np_remainder(pz, L);
        }
        xo[i] = px;
        yo[i] = py;
        zo[i] = pz;
    }
}

int launch_euler_direct_boxes(dem_ctx *ctx, int n, int nbox, const int *off, const double *Lb, const double *x,
                              const double *y, const double *z, const double *r, const double *fx, const double *fy,
                              const double *fz, const double *vx, const double *vy, const double *vz, double stokes,
                              double dt, int periodic, double *xo, double *yo, double *zo, cudaStream_t s) {
    if (n == 0) return DEM_OK;
    const int grid = min(ceil_div(n, 256), 8 * ctx->sm_count);
    euler_direct_boxes_kernel<<<grid, 256, 0, counted(s)>>>(n, nbox, off, Lb, x, y, z, r, fx, fy, fz, vx, vy, vz, stokes,
                                                            dt, periodic, xo, yo, zo);
    return dem_check_launch(ctx, "euler_direct (boxes)");
}

int launch_euler_direct(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                        const double *fx, const double *fy, const double *fz, const double *vx, const double *vy,
                        const double *vz, double stokes, double dt, double L, int periodic, double *xo, double *yo,
                        double *zo, cudaStream_t s) {
    const int grid = min(ceil_div(n, 256), 8 * ctx->sm_count);
    euler_direct_kernel<<<grid, 256, 0, counted(s)>>>(n, x, y, z, r, fx, fy, fz, vx, vy, vz, stokes, dt, L, periodic, xo, yo,
                                             zo);
    return dem_check_launch(ctx, "euler_direct");
}

int launch_euler_total(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *vx,
                       const double *vy, const double *vz, double dt, double L, int periodic, double *xo, double *yo,
                       double *zo, cudaStream_t s) {
    const int grid = min(ceil_div(n, 256), 8 * ctx->sm_count);
    euler_total_kernel<<<grid, 256, 0, counted(s)>>>(n, x, y, z, vx, vy, vz, dt, L, periodic, xo, yo, zo);
    return dem_check_launch(ctx, "euler_total");
}

}  // namespace dem

// ---------------------------------------------------------------------------
// Layout conversion between the reference's (N, 3) row-major arrays and the
// structure-of-arrays layout the kernels use.
// ---------------------------------------------------------------------------
namespace dem {

__global__ void aos_to_soa_kernel(int n, const double *__restrict__ aos, double *__restrict__ x,
                                  double *__restrict__ y, double *__restrict__ z) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = aos[3 * (size_t)i];
        y[i] = aos[3 * (size_t)i + 1];
        z[i] = aos[3 * (size_t)i + 2];
    }
}

__global__ void soa_to_aos_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, double *__restrict__ aos) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        aos[3 * (size_t)i] = x[i];
        aos[3 * (size_t)i + 1] = y[i];
        aos[3 * (size_t)i + 2] = z[i];
    }
}

}  // namespace dem

extern "C" {

int dem_aos_to_soa(dem_ctx *ctx, int n, const double *aos, double *x, double *y, double *z, void *stream) {
    if (!ctx || n < 0) return DEM_E_INVALID;
    if (n == 0) return DEM_OK;
    const int grid = min(ceil_div(n, 256), 8 * ctx->sm_count);
    dem::aos_to_soa_kernel<<<grid, 256, 0, counted((cudaStream_t)stream)>>>(n, aos, x, y, z);
    return dem_check_launch(ctx, "aos_to_soa");
}

int dem_soa_to_aos(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, double *aos, void *stream) {
    if (!ctx || n < 0) return DEM_E_INVALID;
    if (n == 0) return DEM_OK;
    const int grid = min(ceil_div(n, 256), 8 * ctx->sm_count);
    dem::soa_to_aos_kernel<<<grid, 256, 0, counted((cudaStream_t)stream)>>>(n, x, y, z, aos);
    return dem_check_launch(ctx, "soa_to_aos");
}

}  // extern "C"
