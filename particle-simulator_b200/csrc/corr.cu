// corr.cu -- the periodic-image Oseen correction: grid upload and the FP32
// direct pass (the FP64 direct pass is fused into direct_fp64.cu, the tree
// walks take it in tree.cu and bh.cu).
//
// Direct FP32 pass: one thread per target i, j in shared-memory tiles split
// over blockIdx.y; per pair three cell lookups (three 256-bit loads each from
// one 128-byte line; the table, (n-1)^3 x 128 B, stays in L2) and 63 FMA of
// trilinear forms.  Runs of 32 terms
// are summed in FP32 and added in FP64; the j-chunk partials are reduced in a
// fixed order, so results are deterministic.
//
// The grid is not periodic (free-space Stokeslet subtracted), so a pair whose
// minimum image flips changes its term by O(|G| |F_j|), while the sum over j
// cancels to ~1e-3 of the sum of |terms| (the forces sum to zero).  Pairs
// within 1e-6 L of the image boundary on any axis therefore take the image
// decision and the separation from FP64 positions, like the reference.
#include <cmath>
#include <vector>

#include "corr.cuh"

namespace dem {

constexpr int CORR_T = 128;      // threads (targets) per CTA
constexpr int CORR_TILE = 256;   // j per shared-memory tile
constexpr int CORR_SUB = 32;     // terms per FP32 partial: the sums cancel to ~1e-3 of sum |term|

template <bool PER>
__global__ void __launch_bounds__(CORR_T) corr_direct_fp32_kernel(int n, int j_chunk, const double *__restrict__ x,
                                                                  const double *__restrict__ y,
                                                                  const double *__restrict__ z,
                                                                  const double *__restrict__ fx,
                                                                  const double *__restrict__ fy,
                                                                  const double *__restrict__ fz, CorrF32 c,
                                                                  double common, float L, float invL, float edge,
                                                                  float edge_tol, double Ld,
                                                                  double *__restrict__ partial, size_t plane) {
    __shared__ float4 sp[CORR_TILE];  // x, y, z, -
    __shared__ float4 ss[CORR_TILE];  // F_j * common
    const int i = blockIdx.x * CORR_T + threadIdx.x;
    const bool active = i < n;
    const int j0 = blockIdx.y * j_chunk, j1 = min(n, j0 + j_chunk);
    float xi = 0.f, yi = 0.f, zi = 0.f;
    if (active) {
        xi = (float)x[i];
        yi = (float)y[i];
        zi = (float)z[i];
    }
    double Cx = 0.0, Cy = 0.0, Cz = 0.0;
    for (int t0 = j0; t0 < j1; t0 += CORR_TILE) {
        __syncthreads();
        for (int k = threadIdx.x; k < CORR_TILE; k += CORR_T) {
            const int j = t0 + k;
            if (j < j1) {
                sp[k] = make_float4((float)x[j], (float)y[j], (float)z[j], 0.f);
                ss[k] = make_float4((float)(fx[j] * common), (float)(fy[j] * common), (float)(fz[j] * common), 0.f);
            }
        }
        __syncthreads();
        const int cnt = min(CORR_TILE, j1 - t0);
        if (!active) continue;
        for (int k0 = 0; k0 < cnt; k0 += CORR_SUB) {
            float cx = 0.f, cy = 0.f, cz = 0.f;
            const int k1 = min(cnt, k0 + CORR_SUB);
            for (int k = k0; k < k1; ++k) {
                if (t0 + k == i) continue;
                const float4 p = sp[k];
                float dx = xi - p.x, dy = yi - p.y, dz = zi - p.z;
                if (PER) {
                    if (fabsf(fabsf(dx) - edge) < edge_tol || fabsf(fabsf(dy) - edge) < edge_tol ||
                        fabsf(fabsf(dz) - edge) < edge_tol) {  // image decision in FP64 (rare)
                        const int j = t0 + k;
                        const double hL = 0.5 * Ld;
                        dx = (float)mic64(x[i] - x[j], Ld, hL);
                        dy = (float)mic64(y[i] - y[j], Ld, hL);
                        dz = (float)mic64(z[i] - z[j], Ld, hL);
                    } else {  // |d| > L/2 -> d - sign(d) L (positions in [0, L))
                        dx = fmaf(-L, rintf(dx * invL), dx);
                        dy = fmaf(-L, rintf(dy * invL), dy);
                        dz = fmaf(-L, rintf(dz * invL), dz);
                    }
                }
                const float4 s = ss[k];
                corr_pair32(c, dx, dy, dz, s.x, s.y, s.z, cx, cy, cz);
            }
            Cx += (double)cx;
            Cy += (double)cy;
            Cz += (double)cz;
        }
    }
    if (active) {
        double *P = partial + (size_t)blockIdx.y * 3 * plane;
        P[i] = Cx;
        P[plane + i] = Cy;
        P[2 * plane + i] = Cz;
    }
}

// v_i += sum over chunks (in order) + g_self F_i
__global__ void corr_reduce_kernel(int n, int splits, const double *__restrict__ partial, size_t plane,
                                   const double *__restrict__ fx, const double *__restrict__ fy,
                                   const double *__restrict__ fz, double g_self, double *__restrict__ vx,
                                   double *__restrict__ vy, double *__restrict__ vz) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int s = 0; s < splits; ++s) {
            const double *P = partial + (size_t)s * 3 * plane;
            sx += P[i];
            sy += P[plane + i];
            sz += P[2 * plane + i];
        }
        vx[i] += sx + g_self * fx[i];
        vy[i] += sy + g_self * fy[i];
        vz[i] += sz + g_self * fz[i];
    }
}

int launch_corr_direct_fp32(dem_ctx *ctx, const dem_corr *c, int n, const double *x, const double *y,
                            const double *z, const double *fx, const double *fy, const double *fz, double L,
                            int periodic, double *vx, double *vy, double *vz, cudaStream_t s) {
    const int iblocks = ceil_div(n, CORR_T);
    // enough CTAs for ~4 waves at 8 resident CTAs per SM, chunks of whole tiles
    const int want = std::max(1, ceil_div(32LL * ctx->sm_count, iblocks));
    const int j_chunk = ceil_div(ceil_div(n, std::min(want, ceil_div(n, CORR_TILE))), CORR_TILE) * CORR_TILE;
    const int splits = ceil_div(n, j_chunk);
    int rc = dem_ensure_partials(ctx, splits);
    if (rc) return rc;
    const size_t plane = (size_t)ctx->capacity;
    const CorrF32 cf = corr_f32(c, 1.0);
    const float Lf = (float)L, invL = periodic ? (float)(1.0 / L) : 0.f;
    // FP32 separations err by <= ~2 ulp(L) ~ 2.4e-7 L: a margin of 1e-6 L catches every flip
    const float edge = (float)(0.5 * L), edge_tol = (float)(1e-6 * L);
    dem_prof_begin(ctx, "corr_direct_pass", s);
    const dim3 grid(iblocks, splits);
    if (periodic)
        corr_direct_fp32_kernel<true><<<grid, CORR_T, 0, counted(s)>>>(n, j_chunk, x, y, z, fx, fy, fz, cf, c->common,
                                                                       Lf, invL, edge, edge_tol, L, ctx->partial,
                                                                       plane);
    else
        corr_direct_fp32_kernel<false><<<grid, CORR_T, 0, counted(s)>>>(n, j_chunk, x, y, z, fx, fy, fz, cf,
                                                                        c->common, Lf, invL, edge, edge_tol, L,
                                                                        ctx->partial, plane);
    dem_prof_end(ctx, s);
    corr_reduce_kernel<<<std::min(ceil_div(n, 256), 4 * ctx->sm_count), 256, 0, counted(s)>>>(
        n, splits, ctx->partial, plane, fx, fy, fz, c->g_self, vx, vy, vz);
    return dem_check_launch(ctx, "corr_direct_fp32");
}

// Roofline probe: every thread reads `per_thread` cells at pseudo-random
// (xorshift) positions of the FP32 table, 96 bytes each (the three 256-bit
// component loads of one lookup), and writes one sum.
__global__ void corr_gather_probe_kernel(const float *__restrict__ c32, int cells, int per_thread,
                                         float *__restrict__ out) {
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h = tid * 2654435761u + 12345u;
    float acc = 0.f;
    for (int k = 0; k < per_thread; ++k) {
        h ^= h << 13;
        h ^= h >> 17;
        h ^= h << 5;
        const float *p = c32 + (size_t)(h % (uint32_t)cells) * CORR_CELL32;
        float u[8], v[8], w[8];
        corr_ld8(p, u);
        corr_ld8(p + 8, v);
        corr_ld8(p + 16, w);
#pragma unroll
        for (int q = 0; q < 8; ++q) acc += u[q] + v[q] + w[q];
    }
    out[tid] = acc;
}

int launch_direct_convection_fp64_corr(dem_ctx *, const dem_corr *, int, const double *, const double *,
                                       const double *, const double *, const double *, const double *, double,
                                       double, int, double *, double *, double *, cudaStream_t);
int launch_direct_convection_mixed(dem_ctx *, int, const double *, const double *, const double *, const double *,
                                   const double *, const double *, const double *, double, double, int, double *,
                                   double *, double *, cudaStream_t);

}  // namespace dem

// Host: node-major grids -> cell-major FP64 corner blocks and FP32 monomial forms.
static void build_cells(int n, const double *u, const double *v, const double *w, std::vector<double> &c64,
                        std::vector<float> &c32) {
    const size_t m = (size_t)n - 1;
    c64.assign(m * m * m * 24, 0.0);
    c32.assign(m * m * m * CORR_CELL32, 0.f);
    const double *g[3] = {u, v, w};
    for (size_t a = 0; a < m; ++a)
        for (size_t b = 0; b < m; ++b)
            for (size_t d = 0; d < m; ++d) {
                const size_t cell = (a * m + b) * m + d;
                for (int comp = 0; comp < 3; ++comp) {
                    double k[8];
                    for (int q = 0; q < 8; ++q) {
                        const size_t ia = a + (q >> 2), ib = b + ((q >> 1) & 1), id = d + (q & 1);
                        k[q] = g[comp][(ia * n + ib) * n + id];
                        c64[cell * 24 + comp * 8 + q] = k[q];
                    }
                    // f = a0 + t3 a1 + t2 (a2 + t3 a3) + t1 (b0 + t3 b1 + t2 (b2 + t3 b3))
                    const double a0 = k[0], a1 = k[1] - k[0], a2 = k[2] - k[0], a3 = (k[3] - k[2]) - (k[1] - k[0]);
                    const double b0 = k[4] - k[0], b1 = (k[5] - k[4]) - (k[1] - k[0]),
                                 b2 = (k[6] - k[4]) - (k[2] - k[0]),
                                 b3 = ((k[7] - k[6]) - (k[5] - k[4])) - ((k[3] - k[2]) - (k[1] - k[0]));
                    const double coef[8] = {a0, a1, a2, a3, b0, b1, b2, b3};
                    for (int q = 0; q < 8; ++q) c32[cell * CORR_CELL32 + comp * 8 + q] = (float)coef[q];
                }
            }
}

extern "C" {

int dem_corr_create(dem_ctx *ctx, int n, const double *grid_u, const double *grid_v, const double *grid_w,
                    double grid_min, double inv_dx, double Fz_inv, double L_ratio, double eta_ratio,
                    double self_coeff, dem_corr **out) {
    if (!ctx || !out) return DEM_E_INVALID;
    *out = nullptr;
    if (n < 2 || n > DEM_CORR_MAX_GRID)
        return dem_set_error(ctx, DEM_E_INVALID, "correction grid must have 2.." + std::to_string(DEM_CORR_MAX_GRID) +
                                                     " points per axis");
    if (!grid_u || !grid_v || !grid_w) return dem_set_error(ctx, DEM_E_INVALID, "null grid");
    if (!std::isfinite(grid_min) || !std::isfinite(inv_dx) || !(inv_dx > 0) || !std::isfinite(Fz_inv) ||
        !std::isfinite(L_ratio) || !std::isfinite(eta_ratio) || !std::isfinite(self_coeff))
        return dem_set_error(ctx, DEM_E_INVALID, "non-finite correction parameters");
    int rc = dem_check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (rc) return rc;
    std::vector<double> c64;
    std::vector<float> c32;
    build_cells(n, grid_u, grid_v, grid_w, c64, c32);
    dem_corr *c = new dem_corr();
    c->ctx = ctx;
    c->n = n;
    c->gmin = grid_min;
    c->ginv = inv_dx;
    c->Fz_inv = Fz_inv;
    c->cL = L_ratio;
    c->eta_r = eta_ratio;
    c->common = Fz_inv * eta_ratio * L_ratio;  // evaluated left to right, as the reference does per pair
    c->g_self = self_coeff;
    rc = dem_check_cuda(ctx, cudaMalloc((void **)&c->c64, c64.size() * sizeof(double)), "correction grid");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&c->c32, c32.size() * sizeof(float)), "correction grid");
    if (!rc)
        rc = dem_check_cuda(ctx, cudaMemcpy(c->c64, c64.data(), c64.size() * sizeof(double), cudaMemcpyHostToDevice),
                            "correction grid");
    if (!rc)
        rc = dem_check_cuda(ctx, cudaMemcpy(c->c32, c32.data(), c32.size() * sizeof(float), cudaMemcpyHostToDevice),
                            "correction grid");
    if (rc) {
        dem_corr_destroy(c);
        return rc;
    }
    *out = c;
    return DEM_OK;
}

void dem_corr_destroy(dem_corr *c) {
    if (!c) return;
    if (c->ctx) cudaSetDevice(c->ctx->device);
    if (c->c64) cudaFree(c->c64);
    if (c->c32) cudaFree(c->c32);
    delete c;
}

int dem_corr_info(const dem_corr *c, int *n, double *common, double *self_coeff) {
    if (!c) return DEM_E_INVALID;
    if (n) *n = c->n;
    if (common) *common = c->common;
    if (self_coeff) *self_coeff = c->g_self;
    return DEM_OK;
}

int dem_corr_gather_probe(const dem_corr *c, int ctas, int per_thread, float *out, void *stream) {
    if (!c || !out || ctas < 1 || per_thread < 1) return DEM_E_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const int m = c->n - 1;
    dem::corr_gather_probe_kernel<<<ctas, 256, 0, counted(s)>>>(c->c32, m * m * m, per_thread, out);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_E_CUDA;
}

int dem_direct_convection_corr(dem_ctx *ctx, const dem_corr *corr, int n, const double *x, const double *y,
                               const double *z, const double *r, const double *fx, const double *fy, const double *fz,
                               double eta_const, double L, int periodic, int precision, double *vx, double *vy,
                               double *vz, void *stream) {
    if (!ctx) return DEM_E_INVALID;
    if (!corr) return dem_set_error(ctx, DEM_E_NOT_ALLOCATED, "no correction grid loaded");
    if (corr->ctx && corr->ctx->device != ctx->device)
        return dem_set_error(ctx, DEM_E_INVALID, "correction grid lives on another device");
    if (n < 0) return dem_set_error(ctx, DEM_E_INVALID, "n must be >= 0");
    if (n > ctx->capacity) return dem_set_error(ctx, DEM_E_CAPACITY, "number of particles exceeds the capacity");
    if (periodic && !(L > 0)) return dem_set_error(ctx, DEM_E_INVALID, "periodic boundaries need L > 0");
    if (n == 0) return DEM_OK;
    if (!x || !y || !z || !fx || !fy || !fz || !vx || !vy || !vz)
        return dem_set_error(ctx, DEM_E_INVALID, "null pointer");
    int rc = dem_check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == DEM_PREC_FP64)
        return dem::launch_direct_convection_fp64_corr(ctx, corr, n, x, y, z, fx, fy, fz, eta_const, L, periodic, vx,
                                                       vy, vz, s);
    if (precision != DEM_PREC_MIXED) return dem_set_error(ctx, DEM_E_INVALID, "unknown precision");
    if (!r) return dem_set_error(ctx, DEM_E_INVALID, "mixed precision needs the radii");
    rc = dem::launch_direct_convection_mixed(ctx, n, x, y, z, r, fx, fy, fz, eta_const, L, periodic, vx, vy, vz, s);
    if (rc) return rc;
    return dem::launch_corr_direct_fp32(ctx, corr, n, x, y, z, fx, fy, fz, L, periodic, vx, vy, vz, s);
}

}  // extern "C"
