// mixed_common.cuh -- shared pieces of the mixed-precision direct passes
// (direct_mixed.cu: j-split schedule; direct_mixed_sym.cu: symmetric schedule).
#pragma once

#include <cmath>

#include "common.cuh"
#include "tma.cuh"

namespace dem {

constexpr int TJ = 128;    // j per shared-memory tile
constexpr int FLUSH = 64;  // FP32 run length before the compensated fold
constexpr float RINT_MAGIC = 12582912.0f;  // 1.5 * 2^23: (x + M) - M == rint(x) for |x| < 2^22
// Pairs with a separation component within MIC_MARGIN * L of L/2 are sent to
// FP64: FP32 coordinates carry <= ~2^-24 L of rounding, far below this margin.
constexpr double MIC_MARGIN = 1.0 / 262144.0;  // 2^-18

struct MixedArgs {
    int n;
    int j_chunk;  // j per split (multiple of TJ)
    const float4 *pos4;  // (x, y, z, r^3) scaled / (x, y, z, -)
    const float *krf;    // force pass: k_f * r (scaled)
    const float4 *frc4;  // convection pass: (F scaled, k_o * r scaled)
    const double *x, *y, *z, *r;      // FP64 originals
    const double *fx, *fy, *fz;       // FP64 forces (convection pass)
    double L, halfL;
    const unsigned long long *scales;  // [0] max r, [1] max |F| (bit patterns)
    double *partial;  // [splits][3][n]
    uint32_t *err;
};

// Packed FP32x2 arithmetic (sm_100 add/mul/fma.f32x2, round to nearest): one
// instruction on two independent lanes of a float2.
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

__device__ __forceinline__ void two_sum_fold(float &hi, float &lo, float a) {
    const float s = hi + a;
    const float bp = s - hi;
    const float ap = s - bp;
    lo += (hi - ap) + (a - bp);
    hi = s;
}

__device__ __forceinline__ void fold_double(float &hi, float &lo, double v) {
    const float vh = (float)v;
    const float vl = (float)(v - (double)vh);
    two_sum_fold(hi, lo, vh);
    lo += vl;
}

template <bool PER>
__device__ __forceinline__ float mic32(float d, float Ls, float invLs) {
    if (!PER) return d;
    const float u = fmaf(d, invLs, RINT_MAGIC) - RINT_MAGIC;
    return fmaf(-Ls, u, d);
}

// Separation of a pair in FP32 (scaled units).  Returns true when the pair must
// be evaluated exactly in FP64 instead:
//   * near contact: |r_ij| <= k (r_i + r_j) (k folded into ki, kj), which also
//     catches i == j;
//   * periodic image ambiguous in FP32: some |d_axis| within MIC_MARGIN * L of
//     L/2, where FP32 rounding could pick the other image than the reference's
//     FP64 test |d| > L/2 (the pair term is discontinuous there).
template <bool PER, bool FORCE>
__device__ __forceinline__ bool pair_geometry(const float4 &pj, float xi, float yi, float zi, float ki, float kj,
                                              float Ls, float invLs, float hm, float &dx, float &dy, float &dz,
                                              float &r2) {
    if (FORCE) {  // d = x_j - x_i (:229-231)
        dx = pj.x - xi;
        dy = pj.y - yi;
        dz = pj.z - zi;
    } else {  // d = x_i - x_j (:382-384)
        dx = xi - pj.x;
        dy = yi - pj.y;
        dz = zi - pj.z;
    }
    dx = mic32<PER>(dx, Ls, invLs);
    dy = mic32<PER>(dy, Ls, invLs);
    dz = mic32<PER>(dz, Ls, invLs);
    r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float sr = ki + kj;
    bool exact = r2 <= sr * sr;
    if (PER) exact = exact || fabsf(dx) > hm || fabsf(dy) > hm || fabsf(dz) > hm;
    return exact;
}

// FP64 pair terms in scaled units (lengths / ell), reference formulas; L is
// the side of the box the pair lives in.
static __device__ __noinline__ double3 near_force_fp64(int i, int j, const MixedArgs a, int periodic, double inv_ell,
                                                       double L) {
    double3 o = make_double3(0.0, 0.0, 0.0);
    if (i == j) return o;
    double dx = a.x[j] - a.x[i], dy = a.y[j] - a.y[i], dz = a.z[j] - a.z[i];
    if (periodic) {
        dx = mic64(dx, L, 0.5 * L);
        dy = mic64(dy, L, 0.5 * L);
        dz = mic64(dz, L, 0.5 * L);
    }
    const double r_mag = sqrt(dx * dx + dy * dy + dz * dz);
    if (!(r_mag > a.r[i] + a.r[j])) return o;  // contact cut, :246
    const double s = inv_ell;
    dx *= s;
    dy *= s;
    dz *= s;
    const double rm = r_mag * s, rj = a.r[j] * s;
    const double M = ipow3(rj) / ipow7(rm);
    const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
    const double fxy = M * (4 * dz2 - dx2 - dy2);
    o.x = fxy * dx;
    o.y = fxy * dy;
    o.z = M * (2 * dz2 - 3 * dx2 - 3 * dy2) * dz;
    return o;
}

static __device__ __noinline__ double3 near_oseen_fp64(int i, int j, const MixedArgs a, int periodic, double inv_ell,
                                                       double fscale_inv, double L) {
    double3 o = make_double3(0.0, 0.0, 0.0);
    if (i == j) return o;
    double X = a.x[i] - a.x[j], Y = a.y[i] - a.y[j], Z = a.z[i] - a.z[j];
    if (periodic) {
        X = mic64(X, L, 0.5 * L);
        Y = mic64(Y, L, 0.5 * L);
        Z = mic64(Z, L, 0.5 * L);
    }
    const double s = inv_ell;
    X *= s;
    Y *= s;
    Z *= s;
    const double rr = sqrt(X * X + Y * Y + Z * Z);
    const double Fx = a.fx[j] * fscale_inv, Fy = a.fy[j] * fscale_inv, Fz = a.fz[j] * fscale_inv;
    const double inv_r = 1.0 / rr;
    const double inv_r3 = inv_r * inv_r * inv_r;
    const double dot = X * Fx + Y * Fy + Z * Fz;
    o.x = Fx * inv_r + X * dot * inv_r3;
    o.y = Fy * inv_r + Y * dot * inv_r3;
    o.z = Fz * inv_r + Z * dot * inv_r3;
    return o;
}

// 2^-e with 2^(e-1) <= m < 2^e (1 when m == 0 or not finite)
__device__ __forceinline__ double pow2_inv_of(unsigned long long bits) {
    const double m = __longlong_as_double((long long)bits);
    if (!(m > 0.0) || !isfinite(m)) return 1.0;
    int e;
    frexp(m, &e);
    return ldexp(1.0, -e);
}


// ---------------------------------------------------------------------------
// Preparation, scaling and reduction kernels
// ---------------------------------------------------------------------------
// Maximum of |v| over up to three arrays -> slot (as the bit pattern of a
// non-negative double, which orders like an unsigned integer).
static __global__ void maxabs_kernel(int n, const double *__restrict__ a, const double *__restrict__ b,
                              const double *__restrict__ c, unsigned long long *__restrict__ slot) {
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        m = fmax(m, fabs(a[i]));
        if (b) m = fmax(m, fabs(b[i]));
        if (c) m = fmax(m, fabs(c[i]));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(slot, (unsigned long long)__double_as_longlong(m));
}

static __global__ void prep_positions_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                      const double *__restrict__ z, const double *__restrict__ r, double center,
                                      const unsigned long long *__restrict__ scales, double k_near,
                                      float4 *__restrict__ pos4, float *__restrict__ kr) {
    const double s = pow2_inv_of(scales[0]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double rs = r[i] * s;
        pos4[i] = make_float4((float)((x[i] - center) * s), (float)((y[i] - center) * s), (float)((z[i] - center) * s),
                              (float)(rs * rs * rs));
        if (kr) kr[i] = (float)(k_near * rs);
    }
}

static __global__ void prep_forces_kernel(int n, const double *__restrict__ fx, const double *__restrict__ fy,
                                   const double *__restrict__ fz, const double *__restrict__ r,
                                   const unsigned long long *__restrict__ scales, double k_near,
                                   float4 *__restrict__ frc4) {
    const double s = pow2_inv_of(scales[0]);
    const double q = pow2_inv_of(scales[1]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        frc4[i] = make_float4((float)(fx[i] * q), (float)(fy[i] * q), (float)(fz[i] * q), (float)(k_near * r[i] * s));
}

// out_c[i] = factor_i * sum_s partial[s][c][i]
//   force:      factor_i = m_const * (r_i / ell)^3 * ell^2
//   convection: factor   = eta / ell * 2^q
template <bool FORCE>
static __global__ void reduce_partials_kernel(int n, int splits, const double *__restrict__ partial,
                                       const double *__restrict__ r, const unsigned long long *__restrict__ scales,
                                       double coeff, double *__restrict__ ox, double *__restrict__ oy,
                                       double *__restrict__ oz, uint32_t *err) {
    const double s = pow2_inv_of(scales[0]);
    const double ell = 1.0 / s;
    const double q = pow2_inv_of(scales[1]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int p = 0; p < splits; ++p) {
            const double *P = partial + (size_t)p * 3 * n;
            sx += P[i];
            sy += P[n + i];
            sz += P[2 * (size_t)n + i];
        }
        double f;
        if (FORCE) {
            const double rs = r[i] * s;
            f = coeff * ipow3(rs) * ell * ell;
        } else {
            f = coeff * s / q;
        }
        const double vx = f * sx, vy = f * sy, vz = f * sz;
        if (!(isfinite(vx) && isfinite(vy) && isfinite(vz))) raise_device_error(err, DEM_DEVERR_NONFINITE);
        ox[i] = vx;
        oy[i] = vy;
        oz[i] = vz;
    }
}

}  // namespace dem
