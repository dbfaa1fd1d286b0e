// direct_mixed_sym.cu -- mixed-precision direct passes on the symmetric schedule.
//
// The pair force is antisymmetric (the force on j from i is minus the force on
// i from j, direct_droplet_force_calculator.py:183-200) and the Oseen tensor
// is even in d (:401-409), so every unordered pair is evaluated once:
//
//   * droplets are cut into blocks of B = 128 * IPT; a CTA takes one block pair
//     (I, J), I <= J (blockIdx.x enumerates the upper triangle row by row);
//   * I < J: both directions.  The i side accumulates in registers (FP32 runs
//     folded into a compensated (hi, lo) pair, as in direct_mixed.cu).  Over a
//     32-j sub-tile lane l meets j = (l + step) mod 32, so the lanes always
//     hold different j's; each lane adds its j-side terms to the running sum
//     of the j it holds and passes that sum to lane l - 1 (one shuffle per
//     component and half), so after 32 steps every sum is back with the lane
//     owning j;
//   * I == J: ordered pairs, i side only (every i != j pair seen from both ends);
//   * near-contact pairs, i == j and pairs whose periodic image is ambiguous in
//     FP32 are recomputed in FP64 with the reference formula; their j-side
//     terms go to the slot of that j in shared memory (one slot per warp and j);
//   * the per-(I, J) partial sums are written to HBM and added per droplet in a
//     fixed order by reduce_sym_kernel, so results are deterministic.
//
// Arithmetic is packed FP32x2 (sm_100 add/mul/fma.f32x2, round to nearest):
// one instruction evaluates the same j against two i's of the thread, which
// halves the issue slots of the pair terms.  The j tiles are therefore stored
// with every value duplicated, (x, x, y, y), so that they feed the packed
// operands directly; only the comparisons, the rsqrt and the exact-pair
// selects are per element.  Arrays are zero-padded to whole blocks: a padding
// droplet has r^3 = 0 (force) or F = 0 (convection), so its terms vanish and
// no per-pair validity test is needed.
// j-tiles come in by 1-D TMA bulk copies (no multicast) into a double buffer on
// mbarriers with bounded waits, exactly as in the split schedule.
#include "mixed_common.cuh"

namespace dem {

constexpr int SYM_T = 128;  // threads per CTA (4 warps); TJ == SYM_T

__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

// Packed layout of the symmetric passes (npad = nb * B entries, zero padded):
//   force:       p0 = (x, x, y, y)      p1 = (z, z, r^3, r^3)   k2 = (k r, k r)
//   convection:  p0 = -(x, x, y, y)     p1 = (-z, -z, k r, k r)
//                q0 = (Fx, Fx, Fy, Fy)  q1 = (Fz, Fz)
// Coordinates are box-centred and scaled by 1/ell, forces by 2^-q (the scale
// slots); the convection coordinates are stored negated so that d = x_i - x_j
// is one packed add.
struct SymArgs {
    int n, npad, nb, nitems;
    const float4 *p0, *p1, *q0;
    const float2 *k2, *q1;
    MixedArgs m;  // FP64 originals for the exact path
    double *pi;   // [nitems][3][B]  i-side partials
    double *pj;   // [nitems][3][B]  j-side partials (I < J)
};

__host__ __device__ __forceinline__ long long rows_before(long long i, long long nb) {
    return i * nb - (i * (i - 1)) / 2;
}

__device__ __forceinline__ void decode_item(int q, int nb, int &I, int &J) {
    const double b = 2.0 * nb + 1.0;
    int i0 = (int)floor((b - sqrt(b * b - 8.0 * (double)q)) * 0.5);
    if (i0 < 0) i0 = 0;
    if (i0 > nb - 1) i0 = nb - 1;
    while (i0 > 0 && rows_before(i0, nb) > q) --i0;
    while (i0 + 1 < nb && rows_before(i0 + 1, nb) <= q) ++i0;
    I = i0;
    J = I + (int)(q - rows_before(I, nb));
}

template <bool PER>
__device__ __forceinline__ float2 p_mic(float2 d, float2 invL, float2 magic, float2 nmagic, float2 nL) {
    if (!PER) return d;
    const float2 u = p_add(p_fma(d, invL, magic), nmagic);  // rint(d / L)
    return p_fma(nL, u, d);
}

template <bool PER>
__device__ __forceinline__ bool needs_exact(float r2, float sr2, float dx, float dy, float dz, float hm) {
    bool e = r2 <= sr2;
    if (PER) e = e || fabsf(dx) > hm || fabsf(dy) > hm || fabsf(dz) > hm;
    return e;
}

template <int IPT, bool PER, bool FORCE>
__global__ void __launch_bounds__(SYM_T, 4) mixed_sym_kernel(const SymArgs a) {
    static_assert(IPT % 2 == 0, "two i's per packed operation");
    constexpr int B = SYM_T * IPT;
    constexpr int KP = IPT / 2;
    __shared__ __align__(128) float4 s0[2][TJ];
    __shared__ __align__(128) float4 s1[2][TJ];
    __shared__ __align__(128) float4 s2[2][FORCE ? 1 : TJ];
    __shared__ __align__(128) float2 s3[2][TJ];
    __shared__ float jred[SYM_T / 32][3][TJ];
    __shared__ double jnear[SYM_T / 32][3][TJ];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_abort;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = a.n;
    int I, J;
    decode_item(blockIdx.x, a.nb, I, J);
    const bool diag = (I == J);
    const int j0 = J * B;
    constexpr int ntiles = B / TJ;
    const double inv_ell = pow2_inv_of(a.m.scales[0]);
    const double fscale_inv = FORCE ? 1.0 : pow2_inv_of(a.m.scales[1]);
    const float Ls = (float)(a.m.L * inv_ell);
    const float2 invL2 = dup2((float)(1.0 / (a.m.L * inv_ell)));
    const float2 nL2 = dup2(-Ls);
    const float2 magic2 = dup2(RINT_MAGIC), nmagic2 = dup2(-RINT_MAGIC);
    const float hm = (float)(a.m.L * inv_ell * (0.5 - MIC_MARGIN));

    // i state, two i's per packed register: k = 2 kp (.x) and 2 kp + 1 (.y)
    float2 xi[KP], yi[KP], zi[KP], ki[KP], wi[KP];  // force: xi.. = -x_i; wi = r_i^3
    float2 fxi[KP], fyi[KP], fzi[KP];                // convection: F_i
    float2 ax[KP], ay[KP], az[KP];
    float hx[IPT], hy[IPT], hz[IPT], lx[IPT], ly[IPT], lz[IPT];
#pragma unroll
    for (int kp = 0; kp < KP; ++kp) {
        const int ia = I * B + (2 * kp) * SYM_T + tid, ib = ia + SYM_T;
        const float4 a0 = a.p0[ia], b0 = a.p0[ib], a1 = a.p1[ia], b1 = a.p1[ib];
        if (FORCE) {  // d = x_j - x_i: keep -x_i
            xi[kp] = make_float2(-a0.x, -b0.x);
            yi[kp] = make_float2(-a0.z, -b0.z);
            zi[kp] = make_float2(-a1.x, -b1.x);
            wi[kp] = make_float2(a1.z, b1.z);
            ki[kp] = make_float2(a.k2[ia].x, a.k2[ib].x);
        } else {  // d = x_i - x_j, coordinates stored negated: keep +x_i
            xi[kp] = make_float2(-a0.x, -b0.x);
            yi[kp] = make_float2(-a0.z, -b0.z);
            zi[kp] = make_float2(-a1.x, -b1.x);
            ki[kp] = make_float2(a1.z, b1.z);
            const float4 fa = a.q0[ia], fb = a.q0[ib];
            fxi[kp] = make_float2(fa.x, fb.x);
            fyi[kp] = make_float2(fa.z, fb.z);
            fzi[kp] = make_float2(a.q1[ia].x, a.q1[ib].x);
        }
        ax[kp] = ay[kp] = az[kp] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) hx[k] = hy[k] = hz[k] = lx[k] = ly[k] = lz[k] = 0.f;

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbarrier_init();
        s_abort = 0;
    }
    __syncthreads();

    auto issue = [&](int t) {
        const int js = j0 + t * TJ;
        const int b = t & 1;
        constexpr uint32_t b4 = TJ * 16u, b2 = TJ * 8u;
        mbar_arrive_expect_tx(&bar[b], FORCE ? 2 * b4 + b2 : 3 * b4 + b2);
        tma_load_1d(s0[b], a.p0 + js, b4, &bar[b]);
        tma_load_1d(s1[b], a.p1 + js, b4, &bar[b]);
        if (FORCE) {
            tma_load_1d(s3[b], a.k2 + js, b2, &bar[b]);
        } else {
            tma_load_1d(s2[b], a.q0 + js, b4, &bar[b]);
            tma_load_1d(s3[b], a.q1 + js, b2, &bar[b]);
        }
    };

    if (tid == 0) issue(0);
    const size_t plane = (size_t)B;
    double *PJ = a.pj + (size_t)blockIdx.x * 3 * plane;
    bool aborted = false;
    for (int t = 0; t < ntiles; ++t) {
        if (tid == 0 && t + 1 < ntiles) {
            fence_proxy_async_smem();
            issue(t + 1);
        }
        const bool ok = mbar_wait_bounded(&bar[t & 1], (uint32_t)((t >> 1) & 1), a.m.err);
        if (!ok) s_abort = 1;
        const int js = j0 + t * TJ;
        if (ok) {
            const float4 *S0 = s0[t & 1];
            const float4 *S1 = s1[t & 1];
            const float4 *S2 = s2[t & 1];
            const float2 *S3 = s3[t & 1];
            if (!diag)
                for (int q = lane; q < 3 * TJ; q += 32) (&jnear[warp][0][0])[q] = 0.0;
            __syncwarp();
#pragma unroll
            for (int s = 0; s < TJ / 32; ++s) {
                const int jjs = s * 32;
                // Step st: lane l works on j = jjs + (l + st) mod 32.  (sx, sy, sz)
                // is the running j-side sum of the j this lane holds (one half per
                // i of the packed pair); it moves to lane l - 1 after every step.
                float2 sx = make_float2(0.f, 0.f), sy = sx, sz = sx;
#pragma unroll 1
                for (int st = 0; st < 32; ++st) {
                    const int jj = jjs + ((lane + st) & 31);
                    const float4 A = S0[jj], Bv = S1[jj];
                    const float2 pjx = make_float2(A.x, A.y), pjy = make_float2(A.z, A.w);
                    const float2 pjz = make_float2(Bv.x, Bv.y);
                    float2 wj, kj, fjx, fjy, fjz;
                    if (FORCE) {
                        wj = make_float2(Bv.z, Bv.w);
                        kj = S3[jj];
                    } else {
                        kj = make_float2(Bv.z, Bv.w);
                        const float4 Q = S2[jj];
                        fjx = make_float2(Q.x, Q.y);
                        fjy = make_float2(Q.z, Q.w);
                        fjz = S3[jj];
                    }
                    bool ex[IPT];
#pragma unroll
                    for (int kp = 0; kp < KP; ++kp) {
                        float2 dx = p_add(pjx, xi[kp]), dy = p_add(pjy, yi[kp]), dz = p_add(pjz, zi[kp]);
                        dx = p_mic<PER>(dx, invL2, magic2, nmagic2, nL2);
                        dy = p_mic<PER>(dy, invL2, magic2, nmagic2, nL2);
                        dz = p_mic<PER>(dz, invL2, magic2, nmagic2, nL2);
                        const float2 r2 = p_fma(dx, dx, p_fma(dy, dy, p_mul(dz, dz)));
                        const float2 sr = p_add(ki[kp], kj);
                        const float2 sr2 = p_mul(sr, sr);
                        const bool ea = needs_exact<PER>(r2.x, sr2.x, dx.x, dy.x, dz.x, hm);
                        const bool eb = needs_exact<PER>(r2.y, sr2.y, dx.y, dy.y, dz.y, hm);
                        ex[2 * kp] = ea;
                        ex[2 * kp + 1] = eb;
                        float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                        if (FORCE) {
                            // t = -P(d) / r^7 with P the reference's angular factor (:192-199):
                            // P_xy = d_xy (4 dz^2 - dx^2 - dy^2) = -d_xy (r^2 - 5 dz^2),
                            // P_z = dz (2 dz^2 - 3 dx^2 - 3 dy^2) = -dz (r^2 - 5 dz^2 + 2 r^2)
                            const float2 rinv2 = p_mul(rinv, rinv);
                            const float2 rinv4 = p_mul(rinv2, rinv2);
                            float2 base = p_mul(rinv4, p_mul(rinv2, rinv));  // r^-7
                            base.x = ea ? 0.f : base.x;
                            base.y = eb ? 0.f : base.y;
                            const float2 angp = p_fma(p_mul(dup2(-5.f), dz), dz, r2);
                            const float2 angzp = p_fma(dup2(2.f), r2, angp);
                            const float2 gp = p_mul(base, angp);
                            const float2 tx = p_mul(gp, dx), ty = p_mul(gp, dy);
                            const float2 tz = p_mul(p_mul(base, angzp), dz);
                            // i side: sum r_j^3 t = -(force on i) / (m r_i^3); sign restored at the end
                            ax[kp] = p_fma(wj, tx, ax[kp]);
                            ay[kp] = p_fma(wj, ty, ay[kp]);
                            az[kp] = p_fma(wj, tz, az[kp]);
                            if (!diag) {  // force on j: r_i^3 P(-d) / r^7 = r_i^3 t
                                sx = p_fma(wi[kp], tx, sx);
                                sy = p_fma(wi[kp], ty, sy);
                                sz = p_fma(wi[kp], tz, sz);
                            }
                        } else {
                            rinv.x = ea ? 0.f : rinv.x;
                            rinv.y = eb ? 0.f : rinv.y;
                            const float2 rinv2 = p_mul(rinv, rinv);
                            const float2 dot = p_fma(dx, fjx, p_fma(dy, fjy, p_mul(dz, fjz)));
                            const float2 sc = p_mul(dot, rinv2);
                            ax[kp] = p_fma(rinv, p_fma(dx, sc, fjx), ax[kp]);
                            ay[kp] = p_fma(rinv, p_fma(dy, sc, fjy), ay[kp]);
                            az[kp] = p_fma(rinv, p_fma(dz, sc, fjz), az[kp]);
                            if (!diag) {  // velocity at j: the same (even) tensor applied to F_i
                                const float2 doti = p_fma(dx, fxi[kp], p_fma(dy, fyi[kp], p_mul(dz, fzi[kp])));
                                const float2 sci = p_mul(doti, rinv2);
                                sx = p_fma(rinv, p_fma(dx, sci, fxi[kp]), sx);
                                sy = p_fma(rinv, p_fma(dy, sci, fyi[kp]), sy);
                                sz = p_fma(rinv, p_fma(dz, sci, fzi[kp]), sz);
                            }
                        }
                    }
                    bool any = false;
#pragma unroll
                    for (int k = 0; k < IPT; ++k) any |= ex[k];
                    // Rare: exact FP64 terms.  The lanes hold different j's, so
                    // each lane adds its j-side terms to its own j's slot.
                    if (__any_sync(0xffffffffu, any)) {
                        const int j = js + jj;
                        if (any && j < n) {
                            double ex_ = 0.0, ey_ = 0.0, ez_ = 0.0;
#pragma unroll
                            for (int k = 0; k < IPT; ++k) {
                                const int i = I * B + k * SYM_T + tid;
                                if (ex[k] && i < n) {
                                    const double3 v = FORCE ? near_force_fp64(i, j, a.m, PER ? 1 : 0, inv_ell)
                                                            : near_oseen_fp64(i, j, a.m, PER ? 1 : 0, inv_ell,
                                                                              fscale_inv);
                                    const double sg = FORCE ? -1.0 : 1.0;  // the force i side is held negated
                                    fold_double(hx[k], lx[k], sg * v.x);
                                    fold_double(hy[k], ly[k], sg * v.y);
                                    fold_double(hz[k], lz[k], sg * v.z);
                                    if (!diag) {
                                        const double3 w = FORCE
                                                              ? near_force_fp64(j, i, a.m, PER ? 1 : 0, inv_ell)
                                                              : near_oseen_fp64(j, i, a.m, PER ? 1 : 0, inv_ell,
                                                                                fscale_inv);
                                        ex_ += w.x;
                                        ey_ += w.y;
                                        ez_ += w.z;
                                    }
                                }
                            }
                            if (!diag) {
                                jnear[warp][0][jj] += ex_;
                                jnear[warp][1][jj] += ey_;
                                jnear[warp][2][jj] += ez_;
                            }
                        }
                    }
                    if (!diag) {  // pass the running j-side sum to lane - 1
                        const int src = (lane + 1) & 31;
                        sx.x = __shfl_sync(0xffffffffu, sx.x, src);
                        sx.y = __shfl_sync(0xffffffffu, sx.y, src);
                        sy.x = __shfl_sync(0xffffffffu, sy.x, src);
                        sy.y = __shfl_sync(0xffffffffu, sy.y, src);
                        sz.x = __shfl_sync(0xffffffffu, sz.x, src);
                        sz.y = __shfl_sync(0xffffffffu, sz.y, src);
                    }
                }
                if (!diag) {  // the sums are back with the lanes owning their j's
                    jred[warp][0][jjs + lane] = sx.x + sx.y;
                    jred[warp][1][jjs + lane] = sy.x + sy.y;
                    jred[warp][2][jjs + lane] = sz.x + sz.y;
                }
                if (s & 1) {  // fold the FP32 i-side runs every 64 j
#pragma unroll
                    for (int kp = 0; kp < KP; ++kp) {
                        two_sum_fold(hx[2 * kp], lx[2 * kp], ax[kp].x);
                        two_sum_fold(hx[2 * kp + 1], lx[2 * kp + 1], ax[kp].y);
                        two_sum_fold(hy[2 * kp], ly[2 * kp], ay[kp].x);
                        two_sum_fold(hy[2 * kp + 1], ly[2 * kp + 1], ay[kp].y);
                        two_sum_fold(hz[2 * kp], lz[2 * kp], az[kp].x);
                        two_sum_fold(hz[2 * kp + 1], lz[2 * kp + 1], az[kp].y);
                        ax[kp] = ay[kp] = az[kp] = make_float2(0.f, 0.f);
                    }
                }
            }
        }
        __syncthreads();
        if (ok && !diag) {  // combine the warps in a fixed order
            const int lj = t * TJ + tid;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
#pragma unroll
                for (int w = 0; w < SYM_T / 32; ++w) v += (double)jred[w][c][tid] + jnear[w][c][tid];
                PJ[c * plane + lj] = v;
            }
        }
        __syncthreads();
        if (s_abort) {
            aborted = true;
            if (tid == 0 && t + 1 < ntiles) mbar_wait_bounded(&bar[(t + 1) & 1], (uint32_t)(((t + 1) >> 1) & 1), a.m.err);
            break;
        }
    }
    if (aborted) return;
    double *PI = a.pi + (size_t)blockIdx.x * 3 * plane;
    const double sg = FORCE ? -1.0 : 1.0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int li = k * SYM_T + tid;
        PI[li] = sg * ((double)hx[k] + (double)lx[k]);
        PI[plane + li] = sg * ((double)hy[k] + (double)ly[k]);
        PI[2 * plane + li] = sg * ((double)hz[k] + (double)lz[k]);
    }
}

// Packed, zero-padded layout of the symmetric passes (see SymArgs).
template <bool FORCE>
__global__ void prep_sym_kernel(int n, int npad, const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ z, const double *__restrict__ r,
                                const double *__restrict__ fx, const double *__restrict__ fy,
                                const double *__restrict__ fz, double center,
                                const unsigned long long *__restrict__ scales, double k_near, float4 *__restrict__ p0,
                                float4 *__restrict__ p1, float4 *__restrict__ q0, float2 *__restrict__ k2q1) {
    const double s = pow2_inv_of(scales[0]);
    const double q = FORCE ? 1.0 : pow2_inv_of(scales[1]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += gridDim.x * blockDim.x) {
        float X = 0.f, Y = 0.f, Z = 0.f, W = 0.f, K = 0.f, Fx = 0.f, Fy = 0.f, Fz = 0.f;
        if (i < n) {
            const double rs = r[i] * s;
            X = (float)((x[i] - center) * s);
            Y = (float)((y[i] - center) * s);
            Z = (float)((z[i] - center) * s);
            W = (float)(rs * rs * rs);
            K = (float)(k_near * rs);
            if (!FORCE) {
                Fx = (float)(fx[i] * q);
                Fy = (float)(fy[i] * q);
                Fz = (float)(fz[i] * q);
            }
        }
        if (FORCE) {
            p0[i] = make_float4(X, X, Y, Y);
            p1[i] = make_float4(Z, Z, W, W);
            k2q1[i] = make_float2(K, K);
        } else {
            p0[i] = make_float4(-X, -X, -Y, -Y);
            p1[i] = make_float4(-Z, -Z, K, K);
            q0[i] = make_float4(Fx, Fx, Fy, Fy);
            k2q1[i] = make_float2(Fz, Fz);
        }
    }
}

// out_c[d] = factor_d * (sum over items (K, J>=K) of the i side + sum over items (I<K, K) of the j side)
template <bool FORCE>
__global__ void reduce_sym_kernel(int n, int nb, int B, const double *__restrict__ pi, const double *__restrict__ pj,
                                  const double *__restrict__ r, const unsigned long long *__restrict__ scales,
                                  double coeff, double *__restrict__ ox, double *__restrict__ oy,
                                  double *__restrict__ oz, uint32_t *err) {
    const double s = pow2_inv_of(scales[0]);
    const double ell = 1.0 / s;
    const double q = pow2_inv_of(scales[1]);
    const size_t plane = (size_t)B;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const int K = d / B, l = d - K * B;
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int Jb = K; Jb < nb; ++Jb) {
            const double *P = pi + (size_t)(rows_before(K, nb) + (Jb - K)) * 3 * plane;
            sx += P[l];
            sy += P[plane + l];
            sz += P[2 * plane + l];
        }
        for (int Ib = 0; Ib < K; ++Ib) {
            const double *P = pj + (size_t)(rows_before(Ib, nb) + (K - Ib)) * 3 * plane;
            sx += P[l];
            sy += P[plane + l];
            sz += P[2 * plane + l];
        }
        double f;
        if (FORCE) {
            const double rs = r[d] * s;
            f = coeff * ipow3(rs) * ell * ell;
        } else {
            f = coeff * s / q;
        }
        const double vx = f * sx, vy = f * sy, vz = f * sz;
        if (!(isfinite(vx) && isfinite(vy) && isfinite(vz))) raise_device_error(err, DEM_DEVERR_NONFINITE);
        ox[d] = vx;
        oy[d] = vy;
        oz[d] = vz;
    }
}

template <int IPT, bool FORCE>
static void launch_sym(bool per, const SymArgs &a, cudaStream_t s) {
    if (per)
        mixed_sym_kernel<IPT, true, FORCE><<<a.nitems, SYM_T, 0, counted(s)>>>(a);
    else
        mixed_sym_kernel<IPT, false, FORCE><<<a.nitems, SYM_T, 0, counted(s)>>>(a);
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Workspace of the symmetric schedule for n droplets: the packed layout
// (64 bytes per padded droplet) followed by the per-block-pair partial sums.
size_t sym_partial_bytes(int n, int ipt) {
    const long long B = (long long)SYM_T * ipt;
    const long long nb = (n + B - 1) / B;
    const long long items = nb * (nb + 1) / 2;
    return align256((size_t)(nb * B) * 64) + (size_t)(2 * items * 3 * B) * sizeof(double);
}

// Runs the symmetric pass: packs the inputs, evaluates the block pairs and
// reduces per droplet.  The scale slots (max r; max |F| for convection) are
// already filled.  `work` holds sym_partial_bytes(n, ipt) bytes.
template <bool FORCE>
int run_sym_pass(dem_ctx *ctx, int n, int ipt, bool per, const MixedArgs &m, double *work, const double *r,
                 double coeff, double *ox, double *oy, double *oz, cudaStream_t s) {
    ipt = ipt >= 4 ? 4 : 2;
    const int B = SYM_T * ipt;
    const int nb = (n + B - 1) / B;
    const long long items = (long long)nb * (nb + 1) / 2;
    if (items > 0x7fffffffLL) return dem_set_error(ctx, DEM_E_CAPACITY, "symmetric schedule: too many blocks");
    const int npad = nb * B;
    char *base = reinterpret_cast<char *>(work);
    float4 *p0 = reinterpret_cast<float4 *>(base);
    float4 *p1 = p0 + npad;
    float4 *q0 = p1 + npad;
    float2 *k2q1 = reinterpret_cast<float2 *>(q0 + npad);
    const int pgrid = max(1, min(ceil_div(npad, 256), 4 * ctx->sm_count));
    prep_sym_kernel<FORCE><<<pgrid, 256, 0, counted(s)>>>(n, npad, m.x, m.y, m.z, r, m.fx, m.fy, m.fz, 0.5 * m.L,
                                                          m.scales, FORCE ? ctx->tuning.near_force
                                                                          : ctx->tuning.near_oseen,
                                                          p0, p1, q0, k2q1);
    SymArgs a;
    a.n = n;
    a.npad = npad;
    a.nb = nb;
    a.nitems = (int)items;
    a.p0 = p0;
    a.p1 = p1;
    a.q0 = q0;
    a.k2 = k2q1;
    a.q1 = k2q1;
    a.m = m;
    a.pi = reinterpret_cast<double *>(base + align256((size_t)npad * 64));
    a.pj = a.pi + (size_t)items * 3 * B;
    dem_prof_begin(ctx, FORCE ? "mixed_force_pass" : "mixed_convection_pass", s);
    if (ipt == 4)
        launch_sym<4, FORCE>(per, a, s);
    else
        launch_sym<2, FORCE>(per, a, s);
    dem_prof_end(ctx, s);
    int rc = dem_check_launch(ctx, FORCE ? "mixed force (symmetric)" : "mixed convection (symmetric)");
    if (rc) return rc;
    const int rgrid = min(ceil_div(n, 256), 4 * ctx->sm_count);
    reduce_sym_kernel<FORCE><<<rgrid, 256, 0, counted(s)>>>(n, nb, B, a.pi, a.pj, r, m.scales, coeff, ox, oy, oz, ctx->d_err);
    return dem_check_launch(ctx, "mixed reduce (symmetric)");
}

template int run_sym_pass<true>(dem_ctx *, int, int, bool, const MixedArgs &, double *, const double *, double,
                                double *, double *, double *, cudaStream_t);
template int run_sym_pass<false>(dem_ctx *, int, int, bool, const MixedArgs &, double *, const double *, double,
                                 double *, double *, double *, cudaStream_t);

}  // namespace dem
