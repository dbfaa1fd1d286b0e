// capi.cu -- extern "C" entry points (declared in include/dem_b200.h):
// argument validation, capacity checks and dispatch to the kernels.
#include "common.cuh"

namespace dem {
int launch_direct_forces_fp64(dem_ctx *, int, const double *, const double *, const double *, const double *, double,
                              double, int, double *, double *, double *, cudaStream_t);
int launch_direct_convection_fp64(dem_ctx *, int, const double *, const double *, const double *, const double *,
                                  const double *, const double *, double, double, int, double *, double *, double *,
                                  cudaStream_t);
int launch_direct_forces_mixed(dem_ctx *, int, const double *, const double *, const double *, const double *, double,
                               double, int, double *, double *, double *, cudaStream_t);
int launch_direct_convection_mixed(dem_ctx *, int, const double *, const double *, const double *, const double *,
                                   const double *, const double *, const double *, double, double, int, double *,
                                   double *, double *, cudaStream_t);
int launch_euler_direct(dem_ctx *, int, const double *, const double *, const double *, const double *,
                        const double *, const double *, const double *, const double *, const double *,
                        const double *, double, double, double, int, double *, double *, double *, cudaStream_t);
int launch_euler_total(dem_ctx *, int, const double *, const double *, const double *, const double *, const double *,
                       const double *, double, double, int, double *, double *, double *, cudaStream_t);
int launch_hash_detect(dem_ctx *, int, const double *, const double *, const double *, const double *, double, int,
                       int, int32_t *, int64_t, int64_t *, cudaStream_t, int);
int launch_merge(dem_ctx *, int, const double *, const double *, const double *, const double *, const int32_t *,
                 const int64_t *, double *, double *, double *, double *, int32_t *, int32_t *, cudaStream_t);
int launch_direct_vjp(dem_ctx *, int, const double *, const double *, const double *, const double *, const double *,
                      const double *, const double *, const double *, const double *, const double *, double, double,
                      double, double, int, double *, double *, double *, double *, double *, double *, double *,
                      cudaStream_t);
}  // namespace dem

static int check_n(dem_ctx *ctx, int n) {
    if (!ctx) return DEM_E_INVALID;
    if (n < 0) return dem_set_error(ctx, DEM_E_INVALID, "n must be >= 0");
    if (n > ctx->capacity)
        return dem_set_error(ctx, DEM_E_CAPACITY,
                             "number of particles (" + std::to_string(n) + ") exceeds the context capacity (" +
                                 std::to_string(ctx->capacity) + ")");
    return cudaSetDevice(ctx->device) == cudaSuccess ? DEM_OK : dem_set_error(ctx, DEM_E_CUDA, "cudaSetDevice");
}

static int check_box(dem_ctx *ctx, double L, int periodic) {
    if (periodic && !(L > 0)) return dem_set_error(ctx, DEM_E_INVALID, "periodic boundaries need L > 0");
    return DEM_OK;
}

extern "C" {

int dem_direct_forces(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                      double m_const, double L, int periodic, int precision, double *fx, double *fy, double *fz,
                      void *stream) {
    int rc = check_n(ctx, n);
    if (!rc) rc = check_box(ctx, L, periodic);
    if (rc || n == 0) return rc;
    if (!x || !y || !z || !r || !fx || !fy || !fz) return dem_set_error(ctx, DEM_E_INVALID, "null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == DEM_PREC_FP64)
        return dem::launch_direct_forces_fp64(ctx, n, x, y, z, r, m_const, L, periodic, fx, fy, fz, s);
    if (precision == DEM_PREC_MIXED)
        return dem::launch_direct_forces_mixed(ctx, n, x, y, z, r, m_const, L, periodic, fx, fy, fz, s);
    return dem_set_error(ctx, DEM_E_INVALID, "unknown precision");
}

int dem_direct_forces_and_convection(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                                     const double *r, double m_const, double eta_const, double L, int periodic,
                                     int precision, double *fx, double *fy, double *fz, double *vx, double *vy,
                                     double *vz, void *stream) {
    int rc = dem_direct_forces(ctx, n, x, y, z, r, m_const, L, periodic, precision, fx, fy, fz, stream);
    if (rc || n == 0) return rc;
    ctx->sym_reuse_order = precision == DEM_PREC_MIXED;  // the positions are the force pass's
    rc = dem_direct_convection(ctx, n, x, y, z, r, fx, fy, fz, eta_const, L, periodic, precision, vx, vy, vz, stream);
    ctx->sym_reuse_order = false;
    return rc;
}

int dem_direct_convection(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                            const double *fx, const double *fy, const double *fz, double eta_const, double L,
                            int periodic, int precision, double *vx, double *vy, double *vz, void *stream) {
    int rc = check_n(ctx, n);
    if (!rc) rc = check_box(ctx, L, periodic);
    if (rc || n == 0) return rc;
    if (!x || !y || !z || !fx || !fy || !fz || !vx || !vy || !vz)
        return dem_set_error(ctx, DEM_E_INVALID, "null pointer");
    if (precision == DEM_PREC_MIXED && !r) return dem_set_error(ctx, DEM_E_INVALID, "mixed precision needs the radii");
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == DEM_PREC_FP64)
        return dem::launch_direct_convection_fp64(ctx, n, x, y, z, fx, fy, fz, eta_const, L, periodic, vx, vy, vz, s);
    if (precision == DEM_PREC_MIXED)
        return dem::launch_direct_convection_mixed(ctx, n, x, y, z, r, fx, fy, fz, eta_const, L, periodic, vx, vy, vz,
                                                   s);
    return dem_set_error(ctx, DEM_E_INVALID, "unknown precision");
}

int dem_euler_update(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                     const double *fx, const double *fy, const double *fz, const double *vx, const double *vy,
                     const double *vz, double stokes_factor, double dt, double L, int periodic, double *xo,
                     double *yo, double *zo, void *stream) {
    int rc = check_n(ctx, n);
    if (!rc) rc = check_box(ctx, L, periodic);
    if (rc || n == 0) return rc;
    return dem::launch_euler_direct(ctx, n, x, y, z, r, fx, fy, fz, vx, vy, vz, stokes_factor, dt, L, periodic, xo,
                                    yo, zo, (cudaStream_t)stream);
}

int dem_euler_update_total(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *vx,
                           const double *vy, const double *vz, double dt, double L, int periodic, double *xo,
                           double *yo, double *zo, void *stream) {
    int rc = check_n(ctx, n);
    if (!rc) rc = check_box(ctx, L, periodic);
    if (rc || n == 0) return rc;
    return dem::launch_euler_total(ctx, n, x, y, z, vx, vy, vz, dt, L, periodic, xo, yo, zo, (cudaStream_t)stream);
}

int dem_hash_detect(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r, double L,
                    int periodic, int table_size, int32_t *pairs, int64_t pair_capacity, int64_t *counts,
                    void *stream) {
    int rc = check_n(ctx, n);
    if (rc) return rc;
    if (table_size < 1 || (table_size & (table_size - 1)))
        return dem_set_error(ctx, DEM_E_INVALID, "table_size must be a power of two");
    if (!counts || (pair_capacity > 0 && !pairs) || pair_capacity < 0)
        return dem_set_error(ctx, DEM_E_INVALID, "bad pair buffer");
    return dem::launch_hash_detect(ctx, n, x, y, z, r, L, periodic, table_size, pairs, pair_capacity, counts,
                                   (cudaStream_t)stream, 0);
}

int dem_overlap_pairs(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                      double L, int periodic, int table_size, int32_t *pairs, int64_t pair_capacity, int64_t *counts,
                      void *stream) {
    int rc = check_n(ctx, n);
    if (rc) return rc;
    if (!(L > 0)) return dem_set_error(ctx, DEM_E_INVALID, "L must be > 0");
    if (table_size < 1 || (table_size & (table_size - 1)))
        return dem_set_error(ctx, DEM_E_INVALID, "table_size must be a power of two");
    if (!counts || (pair_capacity > 0 && !pairs) || pair_capacity < 0)
        return dem_set_error(ctx, DEM_E_INVALID, "bad pair buffer");
    return dem::launch_hash_detect(ctx, n, x, y, z, r, L, periodic, table_size, pairs, pair_capacity, counts,
                                   (cudaStream_t)stream, 1);
}

int dem_merge(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
              const int32_t *pairs, const int64_t *num_pairs, double *xo, double *yo, double *zo, double *ro,
              int32_t *n_out, int32_t *merged, void *stream) {
    int rc = check_n(ctx, n);
    if (rc) return rc;
    if (!num_pairs || !n_out || !xo || !yo || !zo || !ro) return dem_set_error(ctx, DEM_E_INVALID, "null pointer");
    if (xo == x || yo == y || zo == z || ro == r) return dem_set_error(ctx, DEM_E_INVALID, "outputs alias inputs");
    return dem::launch_merge(ctx, n, x, y, z, r, pairs, num_pairs, xo, yo, zo, ro, n_out, merged,
                             (cudaStream_t)stream);
}

int dem_direct_vjp(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                   const double *fx, const double *fy, const double *fz, const double *lx, const double *ly,
                   const double *lz, double m_const, double eta_const, double stokes_factor, double L, int periodic,
                   double *mx, double *my, double *mz, double *gx, double *gy, double *gz, double *gr, void *stream) {
    int rc = check_n(ctx, n);
    if (rc) return rc;
    if ((rc = check_box(ctx, L, periodic))) return rc;
    if (!(stokes_factor > 0)) return dem_set_error(ctx, DEM_E_INVALID, "stokes_factor must be > 0");
    return dem::launch_direct_vjp(ctx, n, x, y, z, r, fx, fy, fz, lx, ly, lz, m_const, eta_const, stokes_factor, L,
                                  periodic, mx, my, mz, gx, gy, gz, gr, (cudaStream_t)stream);
}

}  // extern "C"
