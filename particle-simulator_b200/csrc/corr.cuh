// corr.cuh -- the periodic-image Oseen correction (COMSOL lattice grid).
//
// The reference adds to every Oseen pair term (and, in the tree walks, to every
// accepted node's monopole) the correction of the periodic images, read from a
// regular n^3 grid of the velocity field of a unit z-force by trilinear
// interpolation; the full tensor comes from three permuted lookups
// (dem/force_calculator/direct_droplet_force_calculator.py:128-182, :413-464;
// dem/octree/flat_tree.py:1070-1131, :1171-1213, :1271-1276):
//
//   xc = d * cL                          (d = MIC(x_i - x_j), cL = L_comsol / L_sim)
//   G_z = (u, v, w)(xc, yc, zc),  G_x = (w, v, u)(zc, yc, xc),  G_y = (u, w, v)(xc, zc, yc)
//   v_i += G_x s_x + G_y s_y + G_z s_z,  s = F_j * (1/Fz_comsol) * eta_ratio * cL
//
// and after the loop the self term g_self * F_i (Stokeslet walks and the
// direct sum only).
//
// Device layout: cell-major.  Cell (a, b, c) of the (n-1)^3 cells holds what
// one lookup needs, so a lookup reads one contiguous block:
//   c64: 24 doubles  u[8] v[8] w[8]   corner values, corner k = (k>>2, (k>>1)&1, k&1)
//   c32: 32 floats   u[8] v[8] w[8] pad[8]   monomial coefficients of the same
//        trilinear form (a0 a1 a2 a3 b0 b1 b2 b3, evaluated by corr_eval32),
//        rounded once from FP64 differences; one 128-byte line per cell, one
//        256-bit load per component
// The FP64 functions restate the reference's expressions in its order and must
// be compiled without multiply-add contraction (-fmad=false).
#pragma once

#include "common.cuh"

struct dem_corr {
    dem_ctx *ctx = nullptr;
    int n = 0;                  // grid points per axis
    double2 *c64 = nullptr;     // (n-1)^3 cells x 12 double2
    float *c32 = nullptr;       // (n-1)^3 cells x 32 floats (128-byte aligned)
    double gmin = 0, ginv = 0;  // first node, 1 / spacing
    double Fz_inv = 0, cL = 0, eta_r = 0;
    double common = 0;          // Fz_inv * eta_r * cL, the reference's per-pair factor
    double g_self = 0;          // self-image coefficient
};

// By-value device view.
struct CorrDev {
    int n;
    const double2 *c64;
    const float *c32;
    double gmin, ginv, cL, common, g_self;
};

static inline CorrDev corr_view(const dem_corr *c) {
    return CorrDev{c->n, c->c64, c->c32, c->gmin, c->ginv, c->cL, c->common, c->g_self};
}

// ---- FP64, the reference's arithmetic ---------------------------------------
// _precompute_grid_idx, direct_droplet_force_calculator.py:146-163, one axis.
__device__ __forceinline__ void corr_axis64(double x, double gmin, double ginv, int n, int &i, double &t) {
    double f = (x - gmin) * ginv;
    const double nmax = (double)(n - 1);
    f = f <= nmax ? f : nmax;  // ti.min(f, n_max)
    f = 0.0 >= f ? 0.0 : f;    // ti.max(0.0, f)
    int k = (int)floor(f);
    k = k <= n - 2 ? k : n - 2;
    i = k;
    t = f - (double)k;
}

// _interp_precomp, :165-182: eight corner terms summed in source order.
__device__ __forceinline__ double corr_interp64(const double (&c)[8], double t1, double t2, double t3) {
    return c[0] * (1 - t1) * (1 - t2) * (1 - t3) + c[1] * (1 - t1) * (1 - t2) * t3 +
           c[2] * (1 - t1) * t2 * (1 - t3) + c[3] * (1 - t1) * t2 * t3 + c[4] * t1 * (1 - t2) * (1 - t3) +
           c[5] * t1 * (1 - t2) * t3 + c[6] * t1 * t2 * (1 - t3) + c[7] * t1 * t2 * t3;
}

__device__ __forceinline__ void corr_cell64(const CorrDev &c, int a, int b, int d, double (&u)[8], double (&v)[8],
                                            double (&w)[8]) {
    const int m = c.n - 1;
    const double2 *p = c.c64 + (((size_t)a * m + b) * m + d) * 12;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double2 qu = __ldg(p + k), qv = __ldg(p + 4 + k), qw = __ldg(p + 8 + k);
        u[2 * k] = qu.x;
        u[2 * k + 1] = qu.y;
        v[2 * k] = qv.x;
        v[2 * k + 1] = qv.y;
        w[2 * k] = qw.x;
        w[2 * k + 1] = qw.y;
    }
}

// One pair (or accepted node): (x, y, z) = MIC(x_i - x_j), F = F_j; adds the
// three components to (vx, vy, vz) the way the reference does, :413-457.
__device__ __forceinline__ void corr_pair64(const CorrDev &c, double x, double y, double z, double Fx, double Fy,
                                            double Fz, double &vx, double &vy, double &vz) {
    const double xc = x * c.cL, yc = y * c.cL, zc = z * c.cL;
    int ax, ay, az;
    double tx, ty, tz;
    corr_axis64(xc, c.gmin, c.ginv, c.n, ax, tx);
    corr_axis64(yc, c.gmin, c.ginv, c.n, ay, ty);
    corr_axis64(zc, c.gmin, c.ginv, c.n, az, tz);
    double u[8], v[8], w[8];
    corr_cell64(c, ax, ay, az, u, v, w);  // G_z at (xc, yc, zc)
    const double gz_x = corr_interp64(u, tx, ty, tz), gz_y = corr_interp64(v, tx, ty, tz),
                 gz_z = corr_interp64(w, tx, ty, tz);
    corr_cell64(c, az, ay, ax, u, v, w);  // G_x at (zc, yc, xc)
    const double gx_x = corr_interp64(w, tz, ty, tx), gx_y = corr_interp64(v, tz, ty, tx),
                 gx_z = corr_interp64(u, tz, ty, tx);
    corr_cell64(c, ax, az, ay, u, v, w);  // G_y at (xc, zc, yc)
    const double gy_x = corr_interp64(u, tx, tz, ty), gy_y = corr_interp64(w, tx, tz, ty),
                 gy_z = corr_interp64(v, tx, tz, ty);
    const double sx = Fx * c.common, sy = Fy * c.common, sz = Fz * c.common;
    vx += gx_x * sx + gy_x * sy + gz_x * sz;
    vy += gx_y * sx + gy_y * sy + gz_y * sz;
    vz += gx_z * sx + gy_z * sy + gz_z * sz;
}

// ---- FP32 (mixed-precision passes and the Morton-tree walk) ------------------
// Grid coordinate f = d * A + B of a separation d in the caller's frame
// (A = scale * cL * ginv, B = -gmin * ginv), clamped like the reference.
constexpr int CORR_CELL32 = 32;  // floats per cell in the FP32 table

struct CorrF32 {
    const float *c32;
    int m;        // cells per axis (n - 1)
    float A, B;   // frame -> grid coordinate
    float fmax;   // n - 1
};

static inline CorrF32 corr_f32(const dem_corr *c, double frame_scale) {
    return CorrF32{c->c32, c->n - 1, (float)(frame_scale * c->cL * c->ginv), (float)(-c->gmin * c->ginv),
                   (float)(c->n - 1)};
}

__device__ __forceinline__ void corr_axis32(const CorrF32 &c, float d, int &i, float &t) {
    const float f = fminf(fmaxf(fmaf(d, c.A, c.B), 0.f), c.fmax);
    const int k = min((int)f, c.m - 1);
    i = k;
    t = f - (float)k;
}

// 32 contiguous bytes (32-byte aligned, read-only for the kernel's lifetime)
// in one 256-bit load.
__device__ __forceinline__ void corr_ld8(const float *p, float (&a)[8]) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(a[4]), "=f"(a[5]), "=f"(a[6]), "=f"(a[7])
        : "l"(p));
}

// a0 + t3 a1 + t2 (a2 + t3 a3) + t1 (b0 + t3 b1 + t2 (b2 + t3 b3)): the trilinear
// form, 7 FMA.
__device__ __forceinline__ float corr_eval32(const float (&c)[8], float t1, float t2, float t3) {
    const float A = fmaf(t2, fmaf(t3, c[3], c[2]), fmaf(t3, c[1], c[0]));
    const float B = fmaf(t2, fmaf(t3, c[7], c[6]), fmaf(t3, c[5], c[4]));
    return fmaf(t1, B, A);
}

// Adds G(d) s to (cx, cy, cz): d = MIC(x_i - x_j) in the caller's frame,
// s = F_j * common in any consistent unit.
__device__ __forceinline__ void corr_pair32(const CorrF32 &c, float dx, float dy, float dz, float sx, float sy,
                                            float sz, float &cx, float &cy, float &cz) {
    int ax, ay, az;
    float tx, ty, tz;
    corr_axis32(c, dx, ax, tx);
    corr_axis32(c, dy, ay, ty);
    corr_axis32(c, dz, az, tz);
    const int m = c.m;
    const float *p1 = c.c32 + ((ax * m + ay) * m + az) * CORR_CELL32;  // G_z at (xc, yc, zc)
    const float *p2 = c.c32 + ((az * m + ay) * m + ax) * CORR_CELL32;  // G_x at (zc, yc, xc)
    const float *p3 = c.c32 + ((ax * m + az) * m + ay) * CORR_CELL32;  // G_y at (xc, zc, yc)
    float u1[8], v1[8], w1[8], u2[8], v2[8], w2[8], u3[8], v3[8], w3[8];
    corr_ld8(p1, u1);
    corr_ld8(p1 + 8, v1);
    corr_ld8(p1 + 16, w1);
    corr_ld8(p2, u2);
    corr_ld8(p2 + 8, v2);
    corr_ld8(p2 + 16, w2);
    corr_ld8(p3, u3);
    corr_ld8(p3 + 8, v3);
    corr_ld8(p3 + 16, w3);
    const float gz_x = corr_eval32(u1, tx, ty, tz), gz_y = corr_eval32(v1, tx, ty, tz),
                gz_z = corr_eval32(w1, tx, ty, tz);
    const float gx_x = corr_eval32(w2, tz, ty, tx), gx_y = corr_eval32(v2, tz, ty, tx),
                gx_z = corr_eval32(u2, tz, ty, tx);
    const float gy_x = corr_eval32(u3, tx, tz, ty), gy_y = corr_eval32(w3, tx, tz, ty),
                gy_z = corr_eval32(v3, tx, tz, ty);
    cx = fmaf(gx_x, sx, fmaf(gy_x, sy, fmaf(gz_x, sz, cx)));
    cy = fmaf(gx_y, sx, fmaf(gy_y, sy, fmaf(gz_y, sz, cy)));
    cz = fmaf(gx_z, sx, fmaf(gy_z, sy, fmaf(gz_z, sz, cz)));
}
