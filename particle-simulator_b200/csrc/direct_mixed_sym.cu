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
//     component), so after 32 steps every sum is back with the lane owning j;
//   * I == J: ordered pairs, i side only (every i != j pair seen from both ends);
//   * near-contact pairs, i == j and pairs whose periodic image is ambiguous in
//     FP32 are recomputed in FP64 with the reference formula; their j-side
//     terms go to the slot of that j in shared memory (one slot per warp and j);
//   * the per-(I, J) partial sums are written to HBM and added per droplet in a
//     fixed order by reduce_sym_kernel, so results are deterministic.
// j-tiles come in by 1-D TMA bulk copies (no multicast) into a double buffer on
// mbarriers with bounded waits, exactly as in the split schedule.
#include "mixed_common.cuh"

namespace dem {

constexpr int SYM_T = 128;  // threads per CTA (4 warps); TJ == SYM_T

struct SymArgs {
    int n, nb, nitems;
    const float4 *pos4;  // (x, y, z, r^3) scaled
    const float *krf;    // force pass: k_f r scaled
    const float4 *frc4;  // convection pass: (F scaled, k_o r scaled)
    MixedArgs m;         // FP64 originals for the exact path
    double *pi;          // [nitems][3][B]  i-side partials
    double *pj;          // [nitems][3][B]  j-side partials (I < J)
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

template <int IPT, bool PER, bool FORCE>
__global__ void __launch_bounds__(SYM_T, 4) mixed_sym_kernel(const SymArgs a) {
    constexpr int B = SYM_T * IPT;
    __shared__ __align__(128) float4 sA[2][TJ];
    __shared__ __align__(128) float4 sB[2][TJ];
    __shared__ __align__(128) float sK[2][TJ];
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
    const int j1 = min(n, j0 + B);
    const int ntiles = j1 > j0 ? (j1 - j0 + TJ - 1) / TJ : 0;
    const double inv_ell = pow2_inv_of(a.m.scales[0]);
    const double fscale_inv = FORCE ? 1.0 : pow2_inv_of(a.m.scales[1]);
    const float Ls = (float)(a.m.L * inv_ell);
    const float invLs = (float)(1.0 / (a.m.L * inv_ell));
    const float hm = (float)(a.m.L * inv_ell * (0.5 - MIC_MARGIN));

    float xi[IPT], yi[IPT], zi[IPT], ki[IPT], wi[IPT];  // wi: r^3 (force) / unused
    float fxi[IPT], fyi[IPT], fzi[IPT];                // convection: F_i scaled
    float ax[IPT], ay[IPT], az[IPT], hx[IPT], hy[IPT], hz[IPT], lx[IPT], ly[IPT], lz[IPT];
    int iidx[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int i = I * B + k * SYM_T + tid;
        iidx[k] = i;
        xi[k] = yi[k] = zi[k] = ki[k] = wi[k] = fxi[k] = fyi[k] = fzi[k] = 0.f;
        if (i < n) {
            const float4 p = a.pos4[i];
            xi[k] = p.x;
            yi[k] = p.y;
            zi[k] = p.z;
            wi[k] = p.w;
            if (FORCE) {
                ki[k] = a.krf[i];
            } else {
                const float4 f = a.frc4[i];
                fxi[k] = f.x;
                fyi[k] = f.y;
                fzi[k] = f.z;
                ki[k] = f.w;
            }
        }
        ax[k] = ay[k] = az[k] = hx[k] = hy[k] = hz[k] = lx[k] = ly[k] = lz[k] = 0.f;
    }

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbarrier_init();
        s_abort = 0;
    }
    __syncthreads();

    auto issue = [&](int t) {
        const int js = j0 + t * TJ;
        const int cnt = min(TJ, j1 - js);
        const int b = t & 1;
        const uint32_t bytes_a = (uint32_t)cnt * 16u;
        if (FORCE) {
            const uint32_t bytes_k = (uint32_t)((cnt + 3) & ~3) * 4u;
            mbar_arrive_expect_tx(&bar[b], bytes_a + bytes_k);
            tma_load_1d(sA[b], a.pos4 + js, bytes_a, &bar[b]);
            tma_load_1d(sK[b], a.krf + js, bytes_k, &bar[b]);
        } else {
            mbar_arrive_expect_tx(&bar[b], 2u * bytes_a);
            tma_load_1d(sA[b], a.pos4 + js, bytes_a, &bar[b]);
            tma_load_1d(sB[b], a.frc4 + js, bytes_a, &bar[b]);
        }
    };

    if (tid == 0 && ntiles > 0) issue(0);
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
        const int cnt = min(TJ, j1 - js);
        if (ok) {
            const float4 *A = sA[t & 1];
            const float4 *Bf = sB[t & 1];
            const float *K = sK[t & 1];
            // j-side sums of the j's this lane owns (j = 32 s + lane of the tile)
            float jx[TJ / 32], jy[TJ / 32], jz[TJ / 32];
#pragma unroll
            for (int s = 0; s < TJ / 32; ++s) jx[s] = jy[s] = jz[s] = 0.f;
            if (!diag)
                for (int q = lane; q < 3 * TJ; q += 32) (&jnear[warp][0][0])[q] = 0.0;
            __syncwarp();
#pragma unroll
            for (int s = 0; s < TJ / 32; ++s) {
                const int jjs = s * 32;
                if (jjs >= cnt) break;
                // Step st: lane l works on j = jjs + (l + st) mod 32, so the 32
                // lanes hold 32 different j's.  (sx, sy, sz) is the running
                // j-side sum of the j this lane holds; it moves to lane l - 1
                // after every step and is back with lane l after 32 steps.
                float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll 1
                for (int st = 0; st < 32; ++st) {
                    const int jj_raw = jjs + ((lane + st) & 31);
                    const bool valid = jj_raw < cnt;
                    const int jj = valid ? jj_raw : jjs;  // a real droplet's data keeps every term finite
                    const float4 pj = A[jj];
                    float4 fj;
                    float kj;
                    if (FORCE) {
                        kj = K[jj];
                    } else {
                        fj = Bf[jj];
                        kj = fj.w;
                    }
                    bool any_exact = false;
#pragma unroll
                    for (int k = 0; k < IPT; ++k) {
                        float dx, dy, dz, r2;
                        const bool exact = pair_geometry<PER, FORCE>(pj, xi[k], yi[k], zi[k], ki[k], kj, Ls, invLs,
                                                                      hm, dx, dy, dz, r2) ||
                                           !valid;
                        any_exact |= exact;
                        float rinv = rsqrtf(r2);
                        if (FORCE) {
                            const float rinv2 = rinv * rinv;
                            const float rinv3 = rinv2 * rinv;
                            const float rinv4 = rinv2 * rinv2;
                            const float base = exact ? 0.f : rinv4 * rinv3;  // r^-7
                            const float ang = fmaf(5.f * dz, dz, -r2);
                            const float angz = fmaf(-2.f, r2, ang);
                            const float g = base * ang;
                            const float tx = g * dx, ty = g * dy, tz = (base * angz) * dz;
                            ax[k] = fmaf(pj.w, tx, ax[k]);  // force on i: r_j^3 P(d) / r^7
                            ay[k] = fmaf(pj.w, ty, ay[k]);
                            az[k] = fmaf(pj.w, tz, az[k]);
                            if (!diag) {  // force on j: - r_i^3 P(d) / r^7
                                sx = fmaf(-wi[k], tx, sx);
                                sy = fmaf(-wi[k], ty, sy);
                                sz = fmaf(-wi[k], tz, sz);
                            }
                        } else {
                            rinv = exact ? 0.f : rinv;
                            const float rinv2 = rinv * rinv;
                            const float dot = fmaf(dx, fj.x, fmaf(dy, fj.y, dz * fj.z));
                            const float sc = dot * rinv2;
                            ax[k] = fmaf(rinv, fmaf(dx, sc, fj.x), ax[k]);
                            ay[k] = fmaf(rinv, fmaf(dy, sc, fj.y), ay[k]);
                            az[k] = fmaf(rinv, fmaf(dz, sc, fj.z), az[k]);
                            if (!diag) {  // velocity at j: same tensor applied to F_i
                                const float doti = fmaf(dx, fxi[k], fmaf(dy, fyi[k], dz * fzi[k]));
                                const float sci = doti * rinv2;
                                sx = fmaf(rinv, fmaf(dx, sci, fxi[k]), sx);
                                sy = fmaf(rinv, fmaf(dy, sci, fyi[k]), sy);
                                sz = fmaf(rinv, fmaf(dz, sci, fzi[k]), sz);
                            }
                        }
                    }
                    // Rare: exact FP64 terms.  The lanes hold different j's, so
                    // each lane adds its j-side terms to its own j's slot.
                    if (__any_sync(0xffffffffu, any_exact)) {
                        if (any_exact && valid) {
                            const int j = js + jj;
                            double ex = 0.0, ey = 0.0, ez = 0.0;
#pragma unroll
                            for (int k = 0; k < IPT; ++k) {
                                float dx, dy, dz, r2;
                                const bool exact = pair_geometry<PER, FORCE>(pj, xi[k], yi[k], zi[k], ki[k], kj, Ls,
                                                                              invLs, hm, dx, dy, dz, r2);
                                if (exact && iidx[k] < n) {
                                    const double3 v = FORCE ? near_force_fp64(iidx[k], j, a.m, PER ? 1 : 0, inv_ell)
                                                            : near_oseen_fp64(iidx[k], j, a.m, PER ? 1 : 0, inv_ell,
                                                                              fscale_inv);
                                    fold_double(hx[k], lx[k], v.x);
                                    fold_double(hy[k], ly[k], v.y);
                                    fold_double(hz[k], lz[k], v.z);
                                    if (!diag) {
                                        const double3 w = FORCE
                                                              ? near_force_fp64(j, iidx[k], a.m, PER ? 1 : 0, inv_ell)
                                                              : near_oseen_fp64(j, iidx[k], a.m, PER ? 1 : 0, inv_ell,
                                                                                fscale_inv);
                                        ex += w.x;
                                        ey += w.y;
                                        ez += w.z;
                                    }
                                }
                            }
                            if (!diag) {
                                jnear[warp][0][jj] += ex;
                                jnear[warp][1][jj] += ey;
                                jnear[warp][2][jj] += ez;
                            }
                        }
                    }
                    if (!diag) {  // pass the running j-side sum to lane - 1
                        const int src = (lane + 1) & 31;
                        sx = __shfl_sync(0xffffffffu, sx, src);
                        sy = __shfl_sync(0xffffffffu, sy, src);
                        sz = __shfl_sync(0xffffffffu, sz, src);
                    }
                }
                if (!diag) {
                    jx[s] = sx;
                    jy[s] = sy;
                    jz[s] = sz;
                }
                if (s & 1) {  // fold the FP32 i-side runs every 64 j
#pragma unroll
                    for (int k = 0; k < IPT; ++k) {
                        two_sum_fold(hx[k], lx[k], ax[k]);
                        two_sum_fold(hy[k], ly[k], ay[k]);
                        two_sum_fold(hz[k], lz[k], az[k]);
                        ax[k] = ay[k] = az[k] = 0.f;
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                two_sum_fold(hx[k], lx[k], ax[k]);
                two_sum_fold(hy[k], ly[k], ay[k]);
                two_sum_fold(hz[k], lz[k], az[k]);
                ax[k] = ay[k] = az[k] = 0.f;
            }
            if (!diag) {
#pragma unroll
                for (int s = 0; s < TJ / 32; ++s) {
                    jred[warp][0][s * 32 + lane] = jx[s];
                    jred[warp][1][s * 32 + lane] = jy[s];
                    jred[warp][2][s * 32 + lane] = jz[s];
                }
            }
        }
        __syncthreads();
        if (ok && !diag && tid < cnt) {  // combine the warps in a fixed order
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
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int li = k * SYM_T + tid;
        PI[li] = (double)hx[k] + (double)lx[k];
        PI[plane + li] = (double)hy[k] + (double)ly[k];
        PI[2 * plane + li] = (double)hz[k] + (double)lz[k];
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

// Bytes of partial sums the symmetric schedule needs for n droplets.
size_t sym_partial_bytes(int n, int ipt) {
    const long long B = (long long)SYM_T * ipt;
    const long long nb = (n + B - 1) / B;
    const long long items = nb * (nb + 1) / 2;
    return (size_t)(2 * items * 3 * B) * sizeof(double);
}

// Runs the symmetric pass; prep kernels have already filled pos4/krf/frc4 and
// the scale slots.  `partial` holds sym_partial_bytes(n, ipt) bytes.
template <bool FORCE>
int run_sym_pass(dem_ctx *ctx, int n, int ipt, bool per, const MixedArgs &m, double *partial, const double *r,
                 double coeff, double *ox, double *oy, double *oz, cudaStream_t s) {
    const int B = SYM_T * ipt;
    const int nb = (n + B - 1) / B;
    const long long items = (long long)nb * (nb + 1) / 2;
    if (items > 0x7fffffffLL) return dem_set_error(ctx, DEM_E_CAPACITY, "symmetric schedule: too many blocks");
    SymArgs a;
    a.n = n;
    a.nb = nb;
    a.nitems = (int)items;
    a.pos4 = m.pos4;
    a.krf = m.krf;
    a.frc4 = m.frc4;
    a.m = m;
    a.pi = partial;
    a.pj = partial + (size_t)items * 3 * B;
    dem_prof_begin(ctx, FORCE ? "mixed_force_pass" : "mixed_convection_pass", s);
    switch (ipt) {
        case 1: launch_sym<1, FORCE>(per, a, s); break;
        case 2: launch_sym<2, FORCE>(per, a, s); break;
        default: launch_sym<4, FORCE>(per, a, s); break;
    }
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
