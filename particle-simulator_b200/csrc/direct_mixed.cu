// direct_mixed.cu -- mixed-precision direct O(N^2) passes for sm_100a.
//
// Pair terms run on the FP32 FMA pipes; FP64 is kept where it matters:
//   * coordinates are rounded to FP32 only after a shift to the box centre and
//     an exact power-of-two rescaling (length unit ell = 2^e ~ max radius), so
//     their absolute error is ~2^-25 of the half box;
//   * every pair with |r_ij| <= k (r_i + r_j) (k = near_force / near_oseen) is
//     recomputed in FP64 from the original coordinates with the reference's
//     exact formula, minimum image and contact cut;
//   * each thread accumulates a j-run of FLUSH terms in FP32, then folds it into
//     a compensated (hi, lo) FP32 pair with Knuth's two-sum; the per-split
//     partials are added in FP64 in a fixed order (deterministic results).
//
// Work decomposition: a CTA owns THREADS*IPT droplets i (IPT register-blocked
// per thread) and one j-chunk (blockIdx.y); j-tiles of packed float4
// (x, y, z, w) are staged in shared memory by 1-D TMA bulk copies into a
// double buffer completed on mbarriers (bounded waits, no multicast), and read
// as warp-wide broadcasts.
//
// Reference: dem/force_calculator/direct_droplet_force_calculator.py:183-253
// (force) and :354-411 (convection).
#include "mixed_common.cuh"

namespace dem {

// ---------------------------------------------------------------------------
// Shared pipeline skeleton: tile t of this CTA's j-chunk lives in buffer t&1.
// ---------------------------------------------------------------------------
template <int IPT, bool PER, bool FORCE>
__global__ void __launch_bounds__(512) mixed_pass_kernel(const MixedArgs a) {
    __shared__ __align__(128) float4 sA[2][TJ];
    __shared__ __align__(128) float4 sB[2][TJ];  // convection: forces; force pass: uses sK
    __shared__ __align__(128) float sK[2][TJ];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_abort;

    const int tid = threadIdx.x, T = blockDim.x;
    const int n = a.n;
    const int ibase = blockIdx.x * T * IPT;
    const int split = blockIdx.y;
    const int j0 = split * a.j_chunk;
    const int j1 = min(n, j0 + a.j_chunk);
    const int ntiles = j1 > j0 ? (j1 - j0 + TJ - 1) / TJ : 0;
    const double inv_ell = pow2_inv_of(a.scales[0]);
    const double fscale_inv = FORCE ? 1.0 : pow2_inv_of(a.scales[1]);
    const float Ls = (float)(a.L * inv_ell);
    const float invLs = (float)(1.0 / (a.L * inv_ell));
    const float hm = (float)(a.L * inv_ell * (0.5 - MIC_MARGIN));

    float xi[IPT], yi[IPT], zi[IPT], ki[IPT];
    float ax[IPT], ay[IPT], az[IPT], hx[IPT], hy[IPT], hz[IPT], lx[IPT], ly[IPT], lz[IPT];
    int iidx[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int i = ibase + k * T + tid;
        iidx[k] = i;
        xi[k] = yi[k] = zi[k] = ki[k] = 0.f;
        if (i < n) {
            const float4 p = a.pos4[i];
            xi[k] = p.x;
            yi[k] = p.y;
            zi[k] = p.z;
            ki[k] = FORCE ? a.krf[i] : a.frc4[i].w;
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
    bool aborted = false;
    for (int t = 0; t < ntiles; ++t) {
        if (tid == 0 && t + 1 < ntiles) {
            fence_proxy_async_smem();
            issue(t + 1);
        }
        const bool ok = mbar_wait_bounded(&bar[t & 1], (uint32_t)((t >> 1) & 1), a.err);
        if (!ok) s_abort = 1;
        if (ok) {
            const int js = j0 + t * TJ;
            const int cnt = min(TJ, j1 - js);
            const float4 *A = sA[t & 1];
            const float4 *B = sB[t & 1];
            const float *K = sK[t & 1];
            for (int jj0 = 0; jj0 < cnt; jj0 += FLUSH) {
                const int jend = min(jj0 + FLUSH, cnt);
#pragma unroll 2
                for (int jj = jj0; jj < jend; ++jj) {
                    const float4 pj = A[jj];
                    float4 fj;
                    float kj;
                    if (FORCE) {
                        kj = K[jj];
                    } else {
                        fj = B[jj];
                        kj = fj.w;
                    }
                    bool any_exact = false;
#pragma unroll
                    for (int k = 0; k < IPT; ++k) {
                        float dx, dy, dz, r2;
                        const bool exact = pair_geometry<PER, FORCE>(pj, xi[k], yi[k], zi[k], ki[k], kj, Ls, invLs,
                                                                      hm, dx, dy, dz, r2);
                        any_exact |= exact;
                        float rinv = rsqrtf(r2);
                        if (FORCE) {
                            const float rinv2 = rinv * rinv;
                            const float rinv3 = rinv2 * rinv;
                            const float rinv4 = rinv2 * rinv2;
                            const float fac = exact ? 0.f : pj.w * (rinv4 * rinv3);
                            const float ang = fmaf(5.f * dz, dz, -r2);  // 4dz^2 - dx^2 - dy^2
                            const float angz = fmaf(-2.f, r2, ang);    // 2dz^2 - 3dx^2 - 3dy^2
                            const float f = fac * ang;
                            ax[k] = fmaf(f, dx, ax[k]);
                            ay[k] = fmaf(f, dy, ay[k]);
                            az[k] = fmaf(fac * angz, dz, az[k]);
                        } else {
                            rinv = exact ? 0.f : rinv;
                            const float rinv2 = rinv * rinv;
                            const float dot = fmaf(dx, fj.x, fmaf(dy, fj.y, dz * fj.z));
                            const float sc = dot * rinv2;
                            ax[k] = fmaf(rinv, fmaf(dx, sc, fj.x), ax[k]);
                            ay[k] = fmaf(rinv, fmaf(dy, sc, fj.y), ay[k]);
                            az[k] = fmaf(rinv, fmaf(dz, sc, fj.z), az[k]);
                        }
                    }
                    // Rare: near-contact pairs, i == j and pairs whose periodic
                    // image is ambiguous in FP32 are evaluated in FP64 with the
                    // reference formula (their FP32 term was zeroed above).
                    if (__any_sync(0xffffffffu, any_exact)) {
                        if (any_exact) {
                            const int j = js + jj;
#pragma unroll
                            for (int k = 0; k < IPT; ++k) {
                                float dx, dy, dz, r2;
                                const bool exact = pair_geometry<PER, FORCE>(pj, xi[k], yi[k], zi[k], ki[k], kj, Ls,
                                                                              invLs, hm, dx, dy, dz, r2);
                                if (exact && iidx[k] < n) {
                                    const double3 v = FORCE ? near_force_fp64(iidx[k], j, a, PER ? 1 : 0, inv_ell, a.L)
                                                            : near_oseen_fp64(iidx[k], j, a, PER ? 1 : 0, inv_ell,
                                                                              fscale_inv, a.L);
                                    fold_double(hx[k], lx[k], v.x);
                                    fold_double(hy[k], ly[k], v.y);
                                    fold_double(hz[k], lz[k], v.z);
                                }
                            }
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
            }
        }
        __syncthreads();
        if (s_abort) {
            aborted = true;
            if (tid == 0 && t + 1 < ntiles) mbar_wait_bounded(&bar[(t + 1) & 1], (uint32_t)(((t + 1) >> 1) & 1), a.err);
            break;
        }
    }
    if (aborted) return;
    const size_t plane = (size_t)n;
    double *P = a.partial + (size_t)split * 3 * plane;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int i = iidx[k];
        if (i < n) {
            P[i] = (double)hx[k] + (double)lx[k];
            P[plane + i] = (double)hy[k] + (double)ly[k];
            P[2 * plane + i] = (double)hz[k] + (double)lz[k];
        }
    }
}

template <int IPT, bool PER, bool FORCE>
static void launch_pass(const MixedArgs &a, dim3 grid, int threads, cudaStream_t s) {
    mixed_pass_kernel<IPT, PER, FORCE><<<grid, threads, 0, counted(s)>>>(a);
}

template <bool FORCE>
static void dispatch_pass(int ipt, bool per, const MixedArgs &a, dim3 grid, int threads, cudaStream_t s) {
    switch (ipt) {
        case 1: per ? launch_pass<1, true, FORCE>(a, grid, threads, s) : launch_pass<1, false, FORCE>(a, grid, threads, s); break;
        case 2: per ? launch_pass<2, true, FORCE>(a, grid, threads, s) : launch_pass<2, false, FORCE>(a, grid, threads, s); break;
        case 8: per ? launch_pass<8, true, FORCE>(a, grid, threads, s) : launch_pass<8, false, FORCE>(a, grid, threads, s); break;
        default: per ? launch_pass<4, true, FORCE>(a, grid, threads, s) : launch_pass<4, false, FORCE>(a, grid, threads, s); break;
    }
}

struct MixedPlan {
    int ipt, threads, splits, j_chunk;
    dim3 grid;
};

template <bool FORCE>
static int resident_ctas(int ipt, bool per, int threads) {
    int occ = 0;
    const void *f = nullptr;
#define DEM_K(I) (per ? (const void *)mixed_pass_kernel<I, true, FORCE> : (const void *)mixed_pass_kernel<I, false, FORCE>)
    switch (ipt) {
        case 1: f = DEM_K(1); break;
        case 2: f = DEM_K(2); break;
        case 8: f = DEM_K(8); break;
        default: f = DEM_K(4); break;
    }
#undef DEM_K
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, threads, 0) != cudaSuccess) occ = 1;
    return occ > 0 ? occ : 1;
}

// Splits the N x N sum into iblocks x splits CTAs.  With j_splits = 0 the
// split count is chosen so that the grid fills whole waves of the resident
// CTA slots (all CTAs do the same work, so a partial last wave idles SMs).
template <bool FORCE>
static MixedPlan plan_for(const dem_ctx *ctx, int n, bool per) {
    MixedPlan p;
    p.ipt = ctx->tuning.i_per_thread;
    p.threads = ctx->tuning.threads;
    const int per_cta = p.threads * p.ipt;
    const int iblocks = ceil_div(n, per_cta);
    const int max_splits = ceil_div(n, TJ);
    auto actual = [&](int s) {
        s = s < 1 ? 1 : (s > max_splits ? max_splits : s);
        const int chunk = ceil_div(ceil_div(n, s), TJ) * TJ;
        return ceil_div(n, chunk);
    };
    int splits = ctx->tuning.j_splits;
    if (splits <= 0) {
        const int slots = resident_ctas<FORCE>(p.ipt, per, p.threads) * ctx->sm_count;
        const int s0 = actual((slots + iblocks - 1) / iblocks);
        double best = -1.0;
        splits = s0;
        for (int s = s0; s <= 8 * s0 && s <= max_splits; ++s) {
            const int sa = actual(s);
            if (sa != s) continue;
            const double waves = (double)iblocks * sa / slots;
            const double eff = waves / std::ceil(waves);
            if (eff > best + 1e-9) {
                best = eff;
                splits = sa;
            }
            if (eff > 0.97) break;
        }
    }
    splits = actual(splits);
    p.j_chunk = ceil_div(ceil_div(n, splits), TJ) * TJ;
    p.splits = ceil_div(n, p.j_chunk);
    p.grid = dim3(iblocks, p.splits, 1);
    return p;
}

size_t sym_partial_bytes(int n, int ipt);
template <bool FORCE>
int run_sym_pass(dem_ctx *ctx, int n, int ipt, bool per, const MixedArgs &m, double *partial, const double *r,
                 double coeff, double *ox, double *oy, double *oz, cudaStream_t s);

// Symmetric schedule: 0 when the split schedule is used, else the i-per-thread
// blocking of the symmetric kernel.  Auto picks the largest blocking (4, then
// 2 rows per thread, at most the tuned i_per_thread) that still gives every SM
// several block pairs -- one CTA per block pair, nb (nb + 1) / 2 of them -- and
// whose partial sums (N^2 / block^2 growth) fit in SYM_BUDGET bytes; with fewer
// block pairs the split schedule, which evaluates every ordered pair but fills
// the GPU, is faster.  Measured on B200 (force + convection pass, N = 1,000 ..
// 65,536): split best to N = 4,096 (sym4 4.3x slower at N = 2,000), sym2 at
// 8,192 - 12,288, sym4 from 16,384 on; the crossovers sit at ~3.5 block pairs
// per SM.
constexpr size_t SYM_BUDGET = size_t(12) << 30;
static long long sym_block_pairs(int n, int ipt) {
    const long long nb = (n + 128LL * ipt - 1) / (128LL * ipt);
    return nb * (nb + 1) / 2;
}
static int symmetric_ipt(const dem_ctx *ctx, int n) {
    const int sched = ctx->tuning.schedule;
    if (sched == DEM_SCHED_SPLIT) return 0;
    const int max_ipt = ctx->tuning.i_per_thread >= 4 ? 4 : 2;  // two i's per packed FP32x2 operation
    if (sched == DEM_SCHED_SYMMETRIC || sched == DEM_SCHED_SYMMETRIC_PLAIN) return max_ipt;
    const long long enough = (long long)(3.5 * ctx->sm_count);
    for (int ipt = max_ipt; ipt >= 2; ipt /= 2)
        if (sym_block_pairs(n, ipt) >= enough && sym_partial_bytes(n, ipt) <= SYM_BUDGET) return ipt;
    return 0;
}

// The plan the mixed passes would run for n droplets (no launch).
int direct_plan(const dem_ctx *ctx, int n, int periodic, int *schedule, int *i_per_thread, int *threads,
                long long *ctas, int *j_splits) {
    const int sym = symmetric_ipt(ctx, n);
    if (sym) {
        const long long B = (long long)128 * sym;
        const long long nb = (n + B - 1) / B;
        *schedule = ctx->tuning.schedule == DEM_SCHED_SYMMETRIC_PLAIN ? DEM_SCHED_SYMMETRIC_PLAIN : DEM_SCHED_SYMMETRIC;
        *i_per_thread = sym;
        *threads = 128;
        *ctas = nb * (nb + 1) / 2;
        *j_splits = 0;
    } else {
        const MixedPlan p = plan_for<true>(ctx, n, periodic != 0);
        *schedule = DEM_SCHED_SPLIT;
        *i_per_thread = p.ipt;
        *threads = p.threads;
        *ctas = (long long)p.grid.x * p.grid.y;
        *j_splits = p.splits;
    }
    return DEM_OK;
}

int launch_direct_forces_mixed(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                               const double *r, double m_const, double L, int periodic, double *fx, double *fy,
                               double *fz, cudaStream_t s) {
    const int sym = symmetric_ipt(ctx, n);
    const MixedPlan p = plan_for<true>(ctx, n, periodic != 0);
    int rc = sym ? dem_ensure_sym_partials(ctx, sym_partial_bytes(n, sym)) : dem_ensure_partials(ctx, p.splits);
    if (rc) return rc;
    unsigned long long *scales = reinterpret_cast<unsigned long long *>(ctx->dscratch);
    rc = dem_check_cuda(ctx, cudaMemsetAsync(scales, 0, 2 * sizeof(unsigned long long), s), "memset");
    if (rc) return rc;
    const int rgrid = min(ceil_div(n, 256), 4 * ctx->sm_count);
    maxabs_kernel<<<rgrid, 256, 0, counted(s)>>>(n, r, nullptr, nullptr, scales);
    float *krf = reinterpret_cast<float *>(ctx->pack_b);  // force pass: k_f r lives in pack_b
    if (!sym)  // the symmetric schedule packs its own layout
        prep_positions_kernel<<<rgrid, 256, 0, counted(s)>>>(n, x, y, z, r, 0.5 * L, scales, ctx->tuning.near_force,
                                                             ctx->pack_a, krf);
    MixedArgs a{};
    a.n = n;
    a.j_chunk = p.j_chunk;
    a.pos4 = ctx->pack_a;
    a.krf = krf;
    a.x = x;
    a.y = y;
    a.z = z;
    a.r = r;
    a.L = L;
    a.halfL = 0.5 * L;
    a.partial = ctx->partial;
    a.err = ctx->d_err;
    a.scales = scales;
    rc = dem_check_launch(ctx, "direct_forces_mixed prep");
    if (rc) return rc;
    if (sym) return run_sym_pass<true>(ctx, n, sym, periodic != 0, a, ctx->sym_partial, r, m_const, fx, fy, fz, s);
    dem_prof_begin(ctx, "mixed_force_pass", s);
    dispatch_pass<true>(p.ipt, periodic != 0, a, p.grid, p.threads, s);
    dem_prof_end(ctx, s);
    rc = dem_check_launch(ctx, "direct_forces_mixed");
    if (rc) return rc;
    reduce_partials_kernel<true><<<rgrid, 256, 0, counted(s)>>>(n, p.splits, ctx->partial, r, scales, m_const, fx, fy, fz,
                                                       ctx->d_err);
    return dem_check_launch(ctx, "direct_forces_mixed reduce");
}

int launch_direct_convection_mixed(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                                   const double *r, const double *fx, const double *fy, const double *fz, double eta,
                                   double L, int periodic, double *vx, double *vy, double *vz, cudaStream_t s) {
    const int sym = symmetric_ipt(ctx, n);
    const MixedPlan p = plan_for<false>(ctx, n, periodic != 0);
    int rc = sym ? dem_ensure_sym_partials(ctx, sym_partial_bytes(n, sym)) : dem_ensure_partials(ctx, p.splits);
    if (rc) return rc;
    unsigned long long *scales = reinterpret_cast<unsigned long long *>(ctx->dscratch);
    rc = dem_check_cuda(ctx, cudaMemsetAsync(scales, 0, 2 * sizeof(unsigned long long), s), "memset");
    if (rc) return rc;
    const int rgrid = min(ceil_div(n, 256), 4 * ctx->sm_count);
    maxabs_kernel<<<rgrid, 256, 0, counted(s)>>>(n, r, nullptr, nullptr, scales);
    maxabs_kernel<<<rgrid, 256, 0, counted(s)>>>(n, fx, fy, fz, scales + 1);
    if (!sym) {  // the symmetric schedule packs its own layout
        prep_positions_kernel<<<rgrid, 256, 0, counted(s)>>>(n, x, y, z, r, 0.5 * L, scales, 0.0, ctx->pack_a,
                                                             nullptr);
        prep_forces_kernel<<<rgrid, 256, 0, counted(s)>>>(n, fx, fy, fz, r, scales, ctx->tuning.near_oseen,
                                                          ctx->pack_b);
    }
    rc = dem_check_launch(ctx, "direct_convection_mixed prep");
    if (rc) return rc;
    MixedArgs a{};
    a.n = n;
    a.j_chunk = p.j_chunk;
    a.pos4 = ctx->pack_a;
    a.frc4 = ctx->pack_b;
    a.x = x;
    a.y = y;
    a.z = z;
    a.r = r;
    a.fx = fx;
    a.fy = fy;
    a.fz = fz;
    a.L = L;
    a.halfL = 0.5 * L;
    a.scales = scales;
    a.partial = ctx->partial;
    a.err = ctx->d_err;
    if (sym) return run_sym_pass<false>(ctx, n, sym, periodic != 0, a, ctx->sym_partial, r, eta, vx, vy, vz, s);
    dem_prof_begin(ctx, "mixed_convection_pass", s);
    dispatch_pass<false>(p.ipt, periodic != 0, a, p.grid, p.threads, s);
    dem_prof_end(ctx, s);
    rc = dem_check_launch(ctx, "direct_convection_mixed");
    if (rc) return rc;
    reduce_partials_kernel<false><<<rgrid, 256, 0, counted(s)>>>(n, p.splits, ctx->partial, r, scales, eta, vx, vy, vz,
                                                        ctx->d_err);
    return dem_check_launch(ctx, "direct_convection_mixed reduce");
}

}  // namespace dem
