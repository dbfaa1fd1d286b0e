// direct_mixed_sym.cu -- mixed-precision direct passes on the symmetric schedule.
//
// The pair force is antisymmetric (the force on j from i is minus the force on
// i from j, direct_droplet_force_calculator.py:183-200) and the Oseen tensor
// is even in d (:401-409), so every unordered pair is evaluated once:
//
//   * droplets are cut into blocks of B = 128 * IPT; a work item is one block
//     pair (I, J), I <= J, of one box (the items of all boxes are numbered
//     consecutively, see sym.cuh);
//   * I < J: both directions.  The i side accumulates in registers (FP32 runs
//     folded into a compensated (hi, lo) pair, as in direct_mixed.cu).  Over a
//     32-j sub-tile lane l meets j = (l + step) mod 32, so the lanes always
//     hold different j's; each lane adds its j-side terms to the running sum
//     of the j it holds and passes that sum to lane l - 1 (one shuffle per
//     component and half), so after 32 steps every sum is back with the lane
//     owning j;
//   * I == J: ordered pairs, i side only (every i != j pair seen from both ends);
//     the j-side sums run there too and are dropped, which keeps the inner
//     loop free of per-item branches (4 % on the convection pass);
//   * near-contact pairs, i == j and pairs whose periodic image is ambiguous in
//     FP32 are recomputed in FP64 with the reference formula; their j-side
//     terms go to the slot of that j in shared memory (one slot per warp and j);
//   * the per-item partial sums are written to HBM and added per droplet in a
//     fixed order by reduce_sym_kernel, so results are deterministic and do
//     not depend on the grid shape.
//
// Arithmetic is packed FP32x2 (sm_100 add/mul/fma.f32x2, round to nearest):
// one instruction evaluates the same j against two i's of the thread, which
// halves the issue slots of the pair terms.  The j tiles are therefore stored
// with every value duplicated, (x, x, y, y), so that they feed the packed
// operands directly; only the comparisons, the rsqrt and the exact-pair
// selects are per element.  Boxes are zero-padded to whole blocks: a padding
// droplet has r^3 = 0 (force) or F = 0 (convection), so its terms vanish and
// no per-pair validity test is needed.
//
// A CTA walks items blockIdx.x, blockIdx.x + gridDim.x, ... (a persistent grid
// when gridDim.x < items).  j-tiles come in by 1-D TMA bulk copies (no
// multicast) into a double buffer on mbarriers with bounded waits; the copy of
// the next tile, possibly of the next item, is in flight while a tile is used.
#include "morton.cuh"
#include "sym.cuh"

namespace dem {

// Packed layout of the symmetric passes (npad_total entries, zero padded):
//   force:       p0 = (x, x, y, y)      p1 = (z, z, r^3, r^3)   k2 = (k r, k r)
//   convection:  p0 = -(x, x, y, y)     p1 = (-z, -z, k r, k r)
//                q0 = (Fx, Fx, Fy, Fy)  q1 = (Fz, Fz)
// Coordinates are centred in their box and scaled by 1/ell_b, forces by
// 2^-q_b (the box's scale slots); the convection coordinates are stored
// negated so that d = x_i - x_j is one packed add.
struct SymArgs {
    SymBoxes t;
    const float4 *p0, *p1, *q0;
    const float2 *k2, *q1;
    MixedArgs m;  // FP64 originals for the exact path
    double *pi;   // [items][3][B]  i-side partials
    double *pj;   // [items][3][B]  j-side partials (I < J)
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

// Processing order of the sorted pair kernel within a box: the nb diagonal
// items (I, I) first, then the off-diagonal items (I < J) row by row.  A
// diagonal item evaluates every ordered pair of a compact block, and most of
// the box's near-contact pairs, which take the FP64 path, lie there: it runs
// several times longer than an off-diagonal item.  Started first, these items
// overlap the rest of the grid instead of forming its tail.
__device__ __forceinline__ void decode_slot(int s, int nb, int &I, int &J) {
    if (s < nb) {
        I = J = s;
        return;
    }
    decode_item(s - nb, nb - 1, I, J);  // upper triangle without the diagonal: rows of nb - 1 - I items
    ++J;
}

// The box of work item q: droplet offset o0 and count n, padded offset p0,
// blocks nbk, side L, scale slots sc; ql = item index within the box.
struct BoxView {
    int o0, n, p0, nbk;
    double L;
    const unsigned long long *sc;
};

__device__ __forceinline__ BoxView item_box(const SymBoxes &t, int B, int q, int &ql) {
    BoxView v;
    if (t.nbox == 1) {
        ql = q;
        v.o0 = 0;
        v.n = t.n1;
        v.p0 = 0;
        v.nbk = t.npad1 / B;
        v.L = t.L1;
        v.sc = t.scales1;
        return v;
    }
    const int b = box_index(t.ioff, t.nbox, q);
    ql = q - t.ioff[b];
    v.o0 = t.off[b];
    v.n = t.off[b + 1] - v.o0;
    v.p0 = t.poff[b];
    v.nbk = (t.poff[b + 1] - v.p0) / B;
    v.L = t.L[b];
    v.sc = t.scales + 2 * b;
    return v;
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
    constexpr int ntiles = B / TJ;
    __shared__ __align__(128) float4 s0[2][TJ];
    __shared__ __align__(128) float4 s1[2][TJ];
    __shared__ __align__(128) float4 s2[2][FORCE ? 1 : TJ];
    __shared__ __align__(128) float2 s3[2][TJ];
    __shared__ float jred[SYM_T / 32][3][TJ];
    __shared__ double jnear[SYM_T / 32][3][TJ];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_abort;

    const int nitems = a.t.items_total;
    if ((int)blockIdx.x >= nitems) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbarrier_init();
        s_abort = 0;
    }
    __syncthreads();

    // j tile t of item q starts at packed index tile_js(q, t)
    auto tile_js = [&](int q, int t) {
        int ql, I, J;
        const BoxView v = item_box(a.t, B, q, ql);
        decode_item(ql, v.nbk, I, J);
        return v.p0 + J * B + t * TJ;
    };
    auto issue = [&](int js, int g) {
        const int b = g & 1;
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

    if (tid == 0) issue(tile_js(blockIdx.x, 0), 0);
    const size_t plane = (size_t)B;
    int g = 0;            // tiles consumed by this CTA (buffer g & 1, phase (g >> 1) & 1)
    bool issued = true;   // tid 0: the copy of tile g is in flight
    for (int q = blockIdx.x; q < nitems; q += gridDim.x) {
        int ql, I, J;
        const BoxView v = item_box(a.t, B, q, ql);
        decode_item(ql, v.nbk, I, J);
        const bool diag = (I == J);
        const double inv_ell = pow2_inv_of(v.sc[0]);
        const double fscale_inv = FORCE ? 1.0 : pow2_inv_of(v.sc[1]);
        const float Ls = (float)(v.L * inv_ell);
        const float2 invL2 = dup2((float)(1.0 / (v.L * inv_ell)));
        const float2 nL2 = dup2(-Ls);
        const float2 magic2 = dup2(RINT_MAGIC), nmagic2 = dup2(-RINT_MAGIC);
        const float hm = (float)(v.L * inv_ell * (0.5 - MIC_MARGIN));

        // i state, two i's per packed register: k = 2 kp (.x) and 2 kp + 1 (.y)
        float2 xi[KP], yi[KP], zi[KP], ki[KP], wi[KP];  // force: xi.. = -x_i; wi = r_i^3
        float2 fxi[KP], fyi[KP], fzi[KP];                // convection: F_i
        float2 ax[KP], ay[KP], az[KP];
        float hx[IPT], hy[IPT], hz[IPT], lx[IPT], ly[IPT], lz[IPT];
#pragma unroll
        for (int kp = 0; kp < KP; ++kp) {
            const int ia = v.p0 + I * B + (2 * kp) * SYM_T + tid, ib = ia + SYM_T;
            const float4 a0 = a.p0[ia], b0 = a.p0[ib], a1 = a.p1[ia], b1 = a.p1[ib];
            // force: d = x_j - x_i, keep -x_i; convection: d = x_i - x_j with the
            // coordinates stored negated, keep +x_i -- both are -p0, -p1
            xi[kp] = make_float2(-a0.x, -b0.x);
            yi[kp] = make_float2(-a0.z, -b0.z);
            zi[kp] = make_float2(-a1.x, -b1.x);
            if (FORCE) {
                wi[kp] = make_float2(a1.z, b1.z);
                ki[kp] = make_float2(a.k2[ia].x, a.k2[ib].x);
            } else {
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
        double *PJ = a.pj + (size_t)q * 3 * plane;

        for (int t = 0; t < ntiles; ++t, ++g) {
            if (tid == 0) {  // prefetch the next tile (of this item or of the next one)
                const int nq = t + 1 < ntiles ? q : q + (int)gridDim.x;
                issued = nq < nitems;
                if (issued) {
                    fence_proxy_async_smem();
                    issue(tile_js(nq, t + 1 < ntiles ? t + 1 : 0), g + 1);
                }
            }
            const bool ok = mbar_wait_bounded(&bar[g & 1], (uint32_t)((g >> 1) & 1), a.m.err);
            if (!ok) s_abort = 1;
            const int jl0 = J * B + t * TJ;  // index of the tile's first j within its box
            if (ok) {
                const float4 *S0 = s0[g & 1];
                const float4 *S1 = s1[g & 1];
                const float4 *S2 = s2[g & 1];
                const float2 *S3 = s3[g & 1];
                if (!diag)
                    for (int c = lane; c < 3 * TJ; c += 32) (&jnear[warp][0][0])[c] = 0.0;
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
                                // force on j: r_i^3 P(-d) / r^7 = r_i^3 t (diagonal items discard it)
                                sx = p_fma(wi[kp], tx, sx);
                                sy = p_fma(wi[kp], ty, sy);
                                sz = p_fma(wi[kp], tz, sz);
                            } else {
                                rinv.x = ea ? 0.f : rinv.x;
                                rinv.y = eb ? 0.f : rinv.y;
                                const float2 rinv2 = p_mul(rinv, rinv);
                                const float2 dot = p_fma(dx, fjx, p_fma(dy, fjy, p_mul(dz, fjz)));
                                const float2 sc = p_mul(dot, rinv2);
                                ax[kp] = p_fma(rinv, p_fma(dx, sc, fjx), ax[kp]);
                                ay[kp] = p_fma(rinv, p_fma(dy, sc, fjy), ay[kp]);
                                az[kp] = p_fma(rinv, p_fma(dz, sc, fjz), az[kp]);
                                {  // velocity at j: the same (even) tensor applied to F_i (diagonal: discarded)
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
                            const int jl = jl0 + jj;  // j within its box
                            if (any && jl < v.n) {
                                const int j = v.o0 + jl;
                                double ex_ = 0.0, ey_ = 0.0, ez_ = 0.0;
#pragma unroll
                                for (int k = 0; k < IPT; ++k) {
                                    const int il = I * B + k * SYM_T + tid;
                                    if (ex[k] && il < v.n) {
                                        const int i = v.o0 + il;
                                        const double3 w1 =
                                            FORCE ? near_force_fp64(i, j, a.m, PER ? 1 : 0, inv_ell, v.L)
                                                  : near_oseen_fp64(i, j, a.m, PER ? 1 : 0, inv_ell, fscale_inv, v.L);
                                        const double sg = FORCE ? -1.0 : 1.0;  // the force i side is held negated
                                        fold_double(hx[k], lx[k], sg * w1.x);
                                        fold_double(hy[k], ly[k], sg * w1.y);
                                        fold_double(hz[k], lz[k], sg * w1.z);
                                        if (!diag) {
                                            const double3 w2 =
                                                FORCE ? near_force_fp64(j, i, a.m, PER ? 1 : 0, inv_ell, v.L)
                                                      : near_oseen_fp64(j, i, a.m, PER ? 1 : 0, inv_ell, fscale_inv,
                                                                        v.L);
                                            ex_ += w2.x;
                                            ey_ += w2.y;
                                            ez_ += w2.z;
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
                        {  // pass the running j-side sum to lane - 1
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
                    double w = 0.0;
#pragma unroll
                    for (int wp = 0; wp < SYM_T / 32; ++wp) w += (double)jred[wp][c][tid] + jnear[wp][c][tid];
                    PJ[c * plane + lj] = w;
                }
            }
            __syncthreads();
            if (s_abort) {  // a copy never arrived: let the one in flight land, then leave
                if (tid == 0 && issued) mbar_wait_bounded(&bar[(g + 1) & 1], (uint32_t)(((g + 1) >> 1) & 1), a.m.err);
                return;
            }
        }
        double *PI = a.pi + (size_t)q * 3 * plane;
        const double sg = FORCE ? -1.0 : 1.0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int li = k * SYM_T + tid;
            PI[li] = sg * ((double)hx[k] + (double)lx[k]);
            PI[plane + li] = sg * ((double)hy[k] + (double)ly[k]);
            PI[2 * plane + li] = sg * ((double)hz[k] + (double)lz[k]);
        }
    }
}

// ---------------------------------------------------------------------------
// Both FP64 terms of one near pair, sharing the square root and the division:
// a on droplet i from j, b on j from i (scaled units, the reference formulas).
// ---------------------------------------------------------------------------
struct NearTerms {
    double ax, ay, az, bx, by, bz;
};

// Force (direct_droplet_force_calculator.py:183-200, 229-249): the term on i is
// r_j^3 g(d), d = x_j - x_i after the minimum image; g is odd in d, so the term
// on j is -r_i^3 g(d).  Both are cut at contact, r <= r_i + r_j.
static __device__ __noinline__ NearTerms near_force_pair_fp64(int i, int j, const MixedArgs a, int periodic,
                                                              double inv_ell, double L) {
    NearTerms o = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double dx = a.x[j] - a.x[i], dy = a.y[j] - a.y[i], dz = a.z[j] - a.z[i];
    if (periodic) {
        dx = mic64(dx, L, 0.5 * L);
        dy = mic64(dy, L, 0.5 * L);
        dz = mic64(dz, L, 0.5 * L);
    }
    const double r_mag = sqrt(dx * dx + dy * dy + dz * dz);
    const double ri = a.r[i], rj = a.r[j];
    if (!(r_mag > ri + rj)) return o;  // contact cut, :246
    const double s = inv_ell;
    dx *= s;
    dy *= s;
    dz *= s;
    const double inv7 = 1.0 / ipow7(r_mag * s);
    const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
    const double fxy = inv7 * (4 * dz2 - dx2 - dy2);
    const double gx = fxy * dx, gy = fxy * dy, gz = inv7 * (2 * dz2 - 3 * dx2 - 3 * dy2) * dz;
    const double cj = ipow3(rj * s), ci = ipow3(ri * s);
    o.ax = cj * gx;
    o.ay = cj * gy;
    o.az = cj * gz;
    o.bx = -ci * gx;
    o.by = -ci * gy;
    o.bz = -ci * gz;
    return o;
}

// Oseen (:381-411, no contact cut): with X = x_i - x_j, the velocity of i from
// F_j is F_j / r + X (X . F_j) / r^3; the tensor is even in X, so j gets the same
// form with F_i.
static __device__ __noinline__ NearTerms near_oseen_pair_fp64(int i, int j, const MixedArgs a, int periodic,
                                                              double inv_ell, double fscale_inv, double L) {
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
    const double inv_r = 1.0 / sqrt(X * X + Y * Y + Z * Z);
    const double inv_r3 = inv_r * inv_r * inv_r;
    const double Fjx = a.fx[j] * fscale_inv, Fjy = a.fy[j] * fscale_inv, Fjz = a.fz[j] * fscale_inv;
    const double Fix = a.fx[i] * fscale_inv, Fiy = a.fy[i] * fscale_inv, Fiz = a.fz[i] * fscale_inv;
    const double dj = (X * Fjx + Y * Fjy + Z * Fjz) * inv_r3, di = (X * Fix + Y * Fiy + Z * Fiz) * inv_r3;
    NearTerms o;
    o.ax = Fjx * inv_r + X * dj;
    o.ay = Fjy * inv_r + Y * dj;
    o.az = Fjz * inv_r + Z * dj;
    o.bx = Fix * inv_r + X * di;
    o.by = Fiy * inv_r + Y * di;
    o.bz = Fiz * inv_r + Z * di;
    return o;
}

// ---------------------------------------------------------------------------
// One box with its droplets in Morton order: lists of far j's without the
// per-pair tests.
//
// The packed layout holds the droplets in Morton order (perm maps a packed
// position to its droplet), so a block of B consecutive positions is compact
// in space (about L/4 per side at N = 65,536).  For a work item (I, J), I < J,
// every j of block J is classified against block I:
//
//   * far: the minimum-image distance from j to the bounding box of block I
//     exceeds k (max r_I + r_j) (0.1 % margin), so no pair of j with block I
//     is near contact;
//   * fixed image on an axis: one periodic image serves every i of the block,
//     with the whole separation interval inside the ambiguity margin; the
//     entry is stored with that image applied on that axis;
//   * unambiguous on an axis that is not fixed: no droplet of block I lies
//     within 2^-17 L (twice the ambiguity margin of the pair test) of the
//     point where its separation from j would be L/2.  Checked against a
//     per-block bitmap of occupied 1/65,536 L bins per axis.
//
// A far j that is unambiguous on every axis gets the mask of its axes that
// are not fixed (0 .. 7); every other j is slow.  The list holds three runs:
//   fast   (mask 0): the loop takes d = x_j - x_i and the pair terms, nothing
//          else; padded to a whole sub-tile with zero-weight entries far away;
//   masked (masks 1 .. 7, in mask order): the loop takes the FP32 minimum
//          image only on the axes of the sub-tile's mask (the OR of its
//          entries' masks, uniform over the CTA), then the pair terms, without
//          the near and ambiguity tests and the FP64 branch; the run is cut to
//          whole sub-tiles and its last entries (< 32) move to the slow run;
//   slow   (the rest, and every j of a diagonal item): the loop of
//          mixed_sym_kernel, padded with zero-weight entries (its near test
//          keeps a padding entry on top of a droplet harmless).
// A far, unambiguous pair is one the slow loop would evaluate in FP32 too, so
// every pair takes the same FP32 / FP64 decision as in mixed_sym_kernel.  All
// warps walk the same lists, so every warp does the same work between the CTA
// barriers.  The j block is classified as it is loaded (coalesced vector loads
// from the L2-resident packed arrays), so it is not staged by TMA.  Results are
// deterministic: lists, sums and their order depend only on the inputs.
// ---------------------------------------------------------------------------
struct SortedArgs {
    SymArgs s;               // packed layout of every box in Morton order
    const int32_t *perm;     // sorted position -> droplet
    const float4 *bounds;    // [blocks][2]: (min s_x, min s_y, min s_z, max k r), (max s_x, max s_y, max s_z, 0)
    const uint32_t *occ;     // [blocks][3][AMB_BINS / 32]: occupied bins of the stored coordinates per block
};

constexpr int SORTED_PAD = 96;      // list slots beyond B: padding of the fast and slow runs (<= 31 each)
constexpr int AMB_BINS = 65536;     // bins per axis of the occupancy bitmaps (a power of two)
constexpr int AMB_WORDS = AMB_BINS / 32;
constexpr int CLS_SLOW = 8;         // classes 0 .. 7: far and unambiguous, with the mask of axes that take the image
constexpr int NCLS = 9;

template <bool FORCE>
constexpr int sorted_entry_bytes() {
    return FORCE ? 16 + 16 + 8 + 4 + 4 + 1 : 16 + 16 + 16 + 8 + 4 + 4 + 1;
}
template <int IPT, bool FORCE>
constexpr int sorted_smem_bytes() {
    return ((SYM_T * IPT + SORTED_PAD) * sorted_entry_bytes<FORCE>() + 15) & ~15;
}

// far entry of the fast run's padding: zero weight, ~10^6 ell from every droplet
constexpr float SORTED_FAR = 1.0e6f;

__device__ __forceinline__ int amb_bin(float v, float Ls, float invLs) {
    return ((int)floorf(fmaf(v, invLs, 0.5f) * (float)AMB_BINS)) & (AMB_BINS - 1);
}

// Class of the stored j entry (sc: coordinates, kj: k r_j) against block I:
// the mask of the axes that take the minimum image (0 .. 7; sc comes back with
// the fixed image applied on the other axes), or CLS_SLOW.
template <bool PER>
__device__ __forceinline__ int classify_j(float sc[3], float kj, const float4 &blo, const float4 &bhi,
                                          const uint32_t *__restrict__ occ, float Ls, float invLs, float hm_fast,
                                          float m_amb) {
    const float lo3[3] = {blo.x, blo.y, blo.z}, hi3[3] = {bhi.x, bhi.y, bhi.z};
    int mask = 0;
    float g2 = 0.f;
    float u3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float dlo = sc[c] - hi3[c], dhi = sc[c] - lo3[c];
        float gap;
        if (PER) {
            const float u = rintf(0.5f * (dlo + dhi) * invLs);
            u3[c] = u;
            dlo = fmaf(-u, Ls, dlo);
            dhi = fmaf(-u, Ls, dhi);
            if (!(dlo >= -hm_fast && dhi <= hm_fast)) mask |= 1 << c;
            // minimum-image distance of the interval from 0: the nearest of its three images
            gap = fmaxf(0.f, fmaxf(dlo, -dhi));
            gap = fminf(gap, fmaxf(0.f, fmaxf(dlo + Ls, -(dhi + Ls))));
            gap = fminf(gap, fmaxf(0.f, fmaxf(dlo - Ls, -(dhi - Ls))));
        } else {
            gap = fmaxf(0.f, fmaxf(dlo, -dhi));
        }
        g2 = fmaf(gap, gap, g2);
    }
    const float kk = blo.w + kj;
    if (!(g2 > 1.001f * kk * kk)) return CLS_SLOW;
    if (!PER) return 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (mask & (1 << c)) {  // a droplet of block I near s_j - L/2 on this axis: ambiguous
            const float a = sc[c] - 0.5f * Ls;
            const int b0 = amb_bin(a - m_amb, Ls, invLs), b1 = amb_bin(a + m_amb, Ls, invLs);
            const uint32_t *w = occ + c * AMB_WORDS;
            if ((w[b0 >> 5] >> (b0 & 31)) & 1u) return CLS_SLOW;
            if ((w[b1 >> 5] >> (b1 & 31)) & 1u) return CLS_SLOW;
        } else {
            sc[c] = fmaf(-u3[c], Ls, sc[c]);
        }
    }
    return mask;
}

// sub-tile loops: MODE_FAST (no image), MODE_MASKED (image on the axes of a uniform mask), MODE_SLOW
enum { MODE_FAST = 0, MODE_MASKED = 1, MODE_SLOW = 2 };

// Near pairs of the slow run (near contact, i == j, ambiguous image) are not
// evaluated where the test finds them.  Each warp queues them (entry code:
// list entry jj | i row k << 10 | owner lane << 12, rows then lanes in order)
// and evaluates the queue 32 pairs at a time, every lane on one pair, once it
// holds more than one sub-tile step can add and at the end of the item.
// Evaluated where found, a pair ran on one lane with the warp waiting on its
// FP64 loads, square root and division; at N = 65,536 a force pass meets
// ~5e5 such pairs (k = 5), a few thousand in every diagonal item.
constexpr int NQ_CAP = 256;  // queued pairs per warp
struct NearQueue {
    uint32_t (*entry)[NQ_CAP];  // [warps][NQ_CAP]
    int *count;                 // [warps]
    double (*mbox)[3][32];      // [warps][3][lane]: the i-side terms of one row and round, per owner lane
};

// Evaluates every queued pair of the calling warp in FP64 (whole warp, uniform
// call).  Terms go to their targets in queue order: within a round the terms
// on one target are added one rank at a time (the pairs' queue order), and
// rounds follow each other.
//   i side: per row k, the sum for each owner lane is handed over in mbox and
//           folded into the owner's compensated sums;
//   j side: an entry of the current sub-tile (cur_sub) collects in jnear
//           (added when the sub-tile writes its partial sums); an earlier
//           entry is added onto its partial sum already written to PJ.
template <int IPT, bool PER, bool FORCE>
__device__ __forceinline__ void near_flush(const SortedArgs &a, const int *CI, const int *CJ, const int *IP, int lane,
                                           int warp, bool diag, const BoxView &v, double inv_ell, double fscale_inv,
                                           int cur_sub, const NearQueue &nq, double (*jnear)[3][32], double *PJ,
                                           float *hx, float *hy, float *hz, float *lx, float *ly, float *lz) {
    constexpr int NW = SYM_T / 32;
    const double sg = FORCE ? -1.0 : 1.0;  // the force i side is held negated
    const unsigned lt = (1u << lane) - 1u;
    const int qn = nq.count[warp];
#pragma unroll 1
    for (int base = 0; base < qn; base += 32) {
        const int s = base + lane;
        int code = -1;
        NearTerms w = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (s < qn) {
            const int c = (int)nq.entry[warp][s];
            const int i = IP[((c >> 10) & 3) * SYM_T + warp * 32 + (c >> 12)], j = CJ[c & 1023];
            if (i >= 0 && j >= 0 && i != j) {  // padding rows and entries (-1) and i == j add nothing
                w = FORCE ? near_force_pair_fp64(i, j, a.s.m, PER ? 1 : 0, inv_ell, v.L)
                          : near_oseen_pair_fp64(i, j, a.s.m, PER ? 1 : 0, inv_ell, fscale_inv, v.L);
                code = c;
            }
        }
        // i side, row by row (static rows: the sums live in registers)
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int key = (code >= 0 && ((code >> 10) & 3) == k) ? (code >> 12) : -1;  // owner lane
            const unsigned owners = __reduce_or_sync(0xffffffffu, key >= 0 ? 1u << key : 0u);
            if (owners == 0u) continue;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            const int rank = __popc(peers & lt);
            const int ranks = (int)__reduce_max_sync(0xffffffffu, key >= 0 ? (unsigned)__popc(peers) : 0u);
            for (int r = 0; r < ranks; ++r) {
                if (key >= 0 && rank == r) {
                    nq.mbox[warp][0][key] = r ? nq.mbox[warp][0][key] + w.ax : w.ax;
                    nq.mbox[warp][1][key] = r ? nq.mbox[warp][1][key] + w.ay : w.ay;
                    nq.mbox[warp][2][key] = r ? nq.mbox[warp][2][key] + w.az : w.az;
                }
                __syncwarp();
            }
            if ((owners >> lane) & 1u) {
                fold_double(hx[k], lx[k], sg * nq.mbox[warp][0][lane]);
                fold_double(hy[k], ly[k], sg * nq.mbox[warp][1][lane]);
                fold_double(hz[k], lz[k], sg * nq.mbox[warp][2][lane]);
            }
            __syncwarp();
        }
        if (!diag) {  // j side (a diagonal item evaluates both orders of each pair on the i side)
            const int key = code >= 0 ? (code & 1023) : -1;  // list entry
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            const int rank = __popc(peers & lt);
            const int ranks = (int)__reduce_max_sync(0xffffffffu, key >= 0 ? (unsigned)__popc(peers) : 0u);
            for (int r = 0; r < ranks; ++r) {
                if (key >= 0 && rank == r) {
                    if ((key >> 5) == cur_sub) {
                        jnear[warp][0][key & 31] += w.bx;
                        jnear[warp][1][key & 31] += w.by;
                        jnear[warp][2][key & 31] += w.bz;
                    } else {
                        double *d = PJ + (size_t)CI[key] * NW * 3;
                        d[0] += w.bx;
                        d[1] += w.by;
                        d[2] += w.bz;
                    }
                }
                __syncwarp();
            }
        }
    }
    if (lane == 0) nq.count[warp] = 0;
    __syncwarp();
}

// Build knobs of the sorted pair kernel: resident CTAs per SM its registers are
// budgeted for, and how the force pass forms r^-7 (1: 2^(-3.5 log2 r^2) from the
// PTX approximate lg2 / ex2, two MUFU operations and one multiply; 0: rsqrt and
// four multiplies).  The relative error of either is below 1e-6.
#ifndef DEM_SORTED_MIN_CTAS
#define DEM_SORTED_MIN_CTAS 4
#endif
#ifndef DEM_FORCE_POW_EXP2
#define DEM_FORCE_POW_EXP2 1
#endif

__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// MASK: the axes that take the minimum image in MODE_MASKED (a compile-time constant, so that a sub-tile
// pays only for its own axes).
template <int IPT, bool PER, bool FORCE, int MODE, int MASK>
__device__ __forceinline__ void sorted_subtile(const SortedArgs &a, const float4 *C0, const float4 *C1,
                                               const float4 *C2, const float2 *C3, const int *CI, const int *CJ,
                                               const int *IP, int e0, int lane, int warp, bool diag,
                                               const BoxView &v,
                                               double inv_ell, double fscale_inv, float2 invL2, float2 magic2,
                                               float2 nmagic2, float2 nL2, float hm, const float2 *xi,
                                               const float2 *yi, const float2 *zi, const float2 *ki,
                                               const float2 *wi, const float2 *fxi, const float2 *fyi,
                                               const float2 *fzi, float2 *ax, float2 *ay, float2 *az, float *hx,
                                               float *hy, float *hz, float *lx, float *ly, float *lz,
                                               double (*jnear)[3][32], const NearQueue &nq, double *PJ,
                                               float2 &sx, float2 &sy, float2 &sz, bool &had_exact) {
    constexpr int B = SYM_T * IPT;
    constexpr int KP = IPT / 2;
    constexpr bool TESTS = MODE == MODE_SLOW;
    constexpr int img = MODE == MODE_SLOW ? 7 : (MODE == MODE_MASKED ? MASK : 0);  // axes that take the image
#pragma unroll 1
    for (int st = 0; st < 32; ++st) {
        const int u = (lane + st) & 31;
        const int jj = e0 + u;
        const float4 A = C0[jj], Bv = C1[jj];
        const float2 pjx = make_float2(A.x, A.y), pjy = make_float2(A.z, A.w);
        const float2 pjz = make_float2(Bv.x, Bv.y);
        float2 wj, kj, fjx, fjy, fjz;
        if (FORCE) {
            wj = make_float2(Bv.z, Bv.w);
            kj = C3[jj];
        } else {
            kj = make_float2(Bv.z, Bv.w);
            const float4 Q = C2[jj];
            fjx = make_float2(Q.x, Q.y);
            fjy = make_float2(Q.z, Q.w);
            fjz = C3[jj];
        }
        bool ex[IPT];
#pragma unroll
        for (int kp = 0; kp < KP; ++kp) {
            float2 dx = p_add(pjx, xi[kp]), dy = p_add(pjy, yi[kp]), dz = p_add(pjz, zi[kp]);
            if (img & 1) dx = p_mic<PER>(dx, invL2, magic2, nmagic2, nL2);
            if (img & 2) dy = p_mic<PER>(dy, invL2, magic2, nmagic2, nL2);
            if (img & 4) dz = p_mic<PER>(dz, invL2, magic2, nmagic2, nL2);
            const float2 dz2 = p_mul(dz, dz);
            const float2 r2 = p_fma(dx, dx, p_fma(dy, dy, dz2));
            bool ea = false, eb = false;
            if (TESTS) {
                const float2 sr = p_add(ki[kp], kj);
                const float2 sr2 = p_mul(sr, sr);
                ea = needs_exact<PER>(r2.x, sr2.x, dx.x, dy.x, dz.x, hm);
                eb = needs_exact<PER>(r2.y, sr2.y, dx.y, dy.y, dz.y, hm);
            }
            ex[2 * kp] = ea;
            ex[2 * kp + 1] = eb;
            if (FORCE) {
#if DEM_FORCE_POW_EXP2
                const float2 e7 = p_mul(dup2(-3.5f), make_float2(lg2_approx(r2.x), lg2_approx(r2.y)));
                float2 base = make_float2(ex2_approx(e7.x), ex2_approx(e7.y));  // r^-7
#else
                const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                const float2 rinv2 = p_mul(rinv, rinv);
                const float2 rinv4 = p_mul(rinv2, rinv2);
                float2 base = p_mul(rinv4, p_mul(rinv2, rinv));  // r^-7
#endif
                if (TESTS) {
                    base.x = ea ? 0.f : base.x;
                    base.y = eb ? 0.f : base.y;
                }
                const float2 angp = p_fma(dz2, dup2(-5.f), r2);  // r^2 - 5 dz^2
                const float2 angzp = p_fma(dup2(2.f), r2, angp);
                const float2 gp = p_mul(base, angp);
                const float2 tx = p_mul(gp, dx), ty = p_mul(gp, dy);
                const float2 tz = p_mul(p_mul(base, angzp), dz);
                ax[kp] = p_fma(wj, tx, ax[kp]);
                ay[kp] = p_fma(wj, ty, ay[kp]);
                az[kp] = p_fma(wj, tz, az[kp]);
                sx = p_fma(wi[kp], tx, sx);
                sy = p_fma(wi[kp], ty, sy);
                sz = p_fma(wi[kp], tz, sz);
            } else {
                float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                if (TESTS) {
                    rinv.x = ea ? 0.f : rinv.x;
                    rinv.y = eb ? 0.f : rinv.y;
                }
                const float2 rinv2 = p_mul(rinv, rinv);
                const float2 dot = p_fma(dx, fjx, p_fma(dy, fjy, p_mul(dz, fjz)));
                const float2 sc = p_mul(dot, rinv2);
                ax[kp] = p_fma(rinv, p_fma(dx, sc, fjx), ax[kp]);
                ay[kp] = p_fma(rinv, p_fma(dy, sc, fjy), ay[kp]);
                az[kp] = p_fma(rinv, p_fma(dz, sc, fjz), az[kp]);
                const float2 doti = p_fma(dx, fxi[kp], p_fma(dy, fyi[kp], p_mul(dz, fzi[kp])));
                const float2 sci = p_mul(doti, rinv2);
                sx = p_fma(rinv, p_fma(dx, sci, fxi[kp]), sx);
                sy = p_fma(rinv, p_fma(dy, sci, fyi[kp]), sy);
                sz = p_fma(rinv, p_fma(dz, sci, fzi[kp]), sz);
            }
        }
        if (TESTS) {
            bool any = false;
#pragma unroll
            for (int k = 0; k < IPT; ++k) any |= ex[k];
            if (__any_sync(0xffffffffu, any)) {  // rare: queue the pairs for the FP64 terms
                const unsigned lt = (1u << lane) - 1u;
                int qn = nq.count[warp];
#pragma unroll
                for (int k = 0; k < IPT; ++k) {
                    const unsigned b = __ballot_sync(0xffffffffu, ex[k]);
                    if (ex[k]) nq.entry[warp][qn + __popc(b & lt)] = (uint32_t)(jj | (k << 10) | (lane << 12));
                    qn += __popc(b);
                }
                __syncwarp();
                if (lane == 0) nq.count[warp] = qn;
                __syncwarp();
                if (qn > NQ_CAP - 32 * IPT) {  // the next step could overflow the queue
                    had_exact = true;          // jnear may hold terms of this sub-tile
                    near_flush<IPT, PER, FORCE>(a, CI, CJ, IP, lane, warp, diag, v, inv_ell, fscale_inv, e0 >> 5, nq,
                                                jnear, PJ, hx, hy, hz, lx, ly, lz);
                }
            }
        }
        {  // pass the running j-side sum to lane - 1
            const int src = (lane + 1) & 31;
            sx.x = __shfl_sync(0xffffffffu, sx.x, src);
            sx.y = __shfl_sync(0xffffffffu, sx.y, src);
            sy.x = __shfl_sync(0xffffffffu, sy.x, src);
            sy.y = __shfl_sync(0xffffffffu, sy.y, src);
            sz.x = __shfl_sync(0xffffffffu, sz.x, src);
            sz.y = __shfl_sync(0xffffffffu, sz.y, src);
        }
    }
}

template <int IPT, bool PER, bool FORCE>
__global__ void __launch_bounds__(SYM_T, DEM_SORTED_MIN_CTAS) mixed_sym_sorted_kernel(const SortedArgs a) {
    static_assert(IPT % 2 == 0, "two i's per packed operation");
    constexpr int B = SYM_T * IPT;
    constexpr int KP = IPT / 2;
    constexpr int CAP = B + SORTED_PAD;
    constexpr int NW = SYM_T / 32;
    static_assert(CAP <= 1024 && IPT <= 4 && NQ_CAP >= 2 * 32 * IPT,
                  "near-pair queue codes: list entry in 10 bits, row in 2; room for one step beyond the threshold");
    extern __shared__ __align__(128) unsigned char sorted_smem[];
    float4 *C0 = reinterpret_cast<float4 *>(sorted_smem);
    float4 *C1 = C0 + CAP;
    float4 *C2 = C1 + CAP;  // convection only
    float2 *C3 = reinterpret_cast<float2 *>(C2 + (FORCE ? 0 : CAP));
    int *CI = reinterpret_cast<int *>(C3 + CAP);  // list entry -> j within block J (-1: padding entry)
    int *CJ = CI + CAP;  // slow-run entry -> its droplet (-1: padding entry or beyond the box)
    unsigned char *CM = reinterpret_cast<unsigned char *>(CJ + CAP);  // list entry -> class (image mask)
    __shared__ double jnear[NW][3][32];           // exact j-side terms of the current sub-tile, per warp
    __shared__ uint32_t nq_entry[NW][NQ_CAP];     // queued near pairs, per warp
    __shared__ int nq_count[NW];
    __shared__ double nq_mbox[NW][3][32];
    __shared__ int IP[B];  // row of block I -> its droplet (-1: beyond the box)
    const NearQueue nq = {nq_entry, nq_count, nq_mbox};
    __shared__ int wcnt[IPT][NW][NCLS];           // entries per round, warp and class
    __shared__ int wpre[IPT][NW][NCLS];           // entries of the class before (round, warp)
    __shared__ int ctot[NCLS], cbase[NCLS];       // entries per class; first entry of a class in the masked run

    const int nitems = a.s.t.items_total;
    if ((int)blockIdx.x >= nitems) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int c = tid; c < NW * 3 * 32; c += SYM_T) (&jnear[0][0][0])[c] = 0.0;
    if (lane == 0) nq_count[warp] = 0;
    const size_t plane = (size_t)B;
    const unsigned lt = (1u << lane) - 1u;

    for (int slot = blockIdx.x; slot < nitems; slot += gridDim.x) {
        // slot: processing order (diagonal items first); q: the item's row-major index, which places its
        // partial sums, so the order changes nothing in the results
        int sl, I, J;
        const BoxView v = item_box(a.s.t, B, slot, sl);
        decode_slot(sl, v.nbk, I, J);
        const int q = slot - sl + (int)(rows_before(I, v.nbk) + (J - I));
        const bool diag = (I == J);
        const double inv_ell = pow2_inv_of(v.sc[0]);
        const double fscale_inv = FORCE ? 1.0 : pow2_inv_of(v.sc[1]);
        const float Ls = (float)(v.L * inv_ell);
        const float invLs = (float)(1.0 / (v.L * inv_ell));
        const float2 invL2 = dup2(invLs);
        const float2 nL2 = dup2(-Ls);
        const float2 magic2 = dup2(RINT_MAGIC), nmagic2 = dup2(-RINT_MAGIC);
        const float hm = (float)(v.L * inv_ell * (0.5 - MIC_MARGIN));
        // fast intervals and the bitmap check keep another MIC_MARGIN from the pair test's margin
        // (FP32 rounding of the bounds and bins is ~2^-22 L)
        const float hm_fast = (float)(v.L * inv_ell * (0.5 - 2.0 * MIC_MARGIN));
        const float m_amb = (float)(v.L * inv_ell * 2.0 * MIC_MARGIN);

        // ---- the lists of block J against block I: count per class, then write ----
        const int gI = v.p0 / B + I;  // block I of this box in the table of all blocks
        const float4 blo = a.bounds[2 * gI], bhi = a.bounds[2 * gI + 1];
        const uint32_t *occ = a.occ + (size_t)gI * 3 * AMB_WORDS;
        auto load_entry = [&](int p, float4 &A, float4 &Bv, float4 &Q, float2 &S3) {
            A = a.s.p0[p];
            Bv = a.s.p1[p];
            Q = FORCE ? make_float4(0.f, 0.f, 0.f, 0.f) : a.s.q0[p];
            S3 = FORCE ? a.s.k2[p] : a.s.q1[p];
        };
        auto class_of = [&](const float4 &A, const float4 &Bv, const float2 &S3, float sc[3]) {
            sc[0] = A.x;
            sc[1] = A.z;
            sc[2] = Bv.x;
            if (diag) return (int)CLS_SLOW;
            return classify_j<PER>(sc, FORCE ? S3.x : Bv.z, blo, bhi, occ, Ls, invLs, hm_fast, m_amb);
        };
        for (int c = tid; c < IPT * NW * NCLS; c += SYM_T) (&wcnt[0][0][0])[c] = 0;
        __syncthreads();
#pragma unroll 1
        for (int k = 0; k < IPT; ++k) {  // pass 1: entries per (round, warp, class)
            float4 A, Bv, Q;
            float2 S3;
            float sc[3];
            load_entry(v.p0 + J * B + k * SYM_T + tid, A, Bv, Q, S3);
            const int cls = class_of(A, Bv, S3, sc);
            const unsigned peers = __match_any_sync(0xffffffffu, cls);
            if ((peers & lt) == 0) wcnt[k][warp][cls] = __popc(peers);
        }
        __syncthreads();
        if (tid < NCLS) {  // per class: the entries before each (round, warp), and the total
            int acc = 0;
            for (int k = 0; k < IPT; ++k)
                for (int w = 0; w < NW; ++w) {
                    wpre[k][w][tid] = acc;
                    acc += wcnt[k][w][tid];
                }
            ctot[tid] = acc;
        }
        __syncthreads();
        if (tid == 0) {  // the masked run holds masks 1 .. 7 in mask order
            int acc = 0;
            for (int c = 1; c < CLS_SLOW; ++c) {
                cbase[c] = acc;
                acc += ctot[c];
            }
            cbase[0] = acc;  // (the masked run's length)
        }
        __syncthreads();
        const int nA = ctot[0], A_pad = (nA + 31) & ~31;    // fast run, padded
        const int nB = cbase[0], B_used = nB & ~31;          // masked run, cut to whole sub-tiles
        const int nS = ctot[CLS_SLOW];
        const int C_len = nS + (nB - B_used), C_pad = (C_len + 31) & ~31;  // slow run (+ the cut entries)
        const int C0e = A_pad + B_used;                      // first entry of the slow run
#pragma unroll 1
        for (int k = 0; k < IPT; ++k) {  // pass 2: every entry to its place
            float4 A, Bv, Q;
            float2 S3;
            float sc[3];
            const int jb = k * SYM_T + tid;
            load_entry(v.p0 + J * B + jb, A, Bv, Q, S3);
            const int cls = class_of(A, Bv, S3, sc);
            const unsigned peers = __match_any_sync(0xffffffffu, cls);
            const int rank = wpre[k][warp][cls] + __popc(peers & lt);
            int e;
            if (cls == 0) {
                e = rank;
            } else if (cls < CLS_SLOW) {
                const int rb = cbase[cls] + rank;
                e = rb < B_used ? A_pad + rb : C0e + nS + (rb - B_used);
            } else {
                e = C0e + rank;
            }
            if (cls < CLS_SLOW) {  // the fixed images of the entry's unmasked axes
                A = make_float4(sc[0], sc[0], sc[1], sc[1]);
                Bv.x = Bv.y = sc[2];
            }
            C0[e] = A;
            C1[e] = Bv;
            if (!FORCE) C2[e] = Q;
            C3[e] = S3;
            CI[e] = jb;
            if (e >= C0e) CJ[e] = J * B + jb < v.n ? a.perm[v.o0 + J * B + jb] : -1;  // near pairs: slow run only
            CM[e] = (unsigned char)cls;
        }
        // padding: the fast run's lies far from every droplet, the slow run's at the centre; zero weight
        if (tid < 64) {
            const bool fast_pad = tid < 32;
            const int e = fast_pad ? nA + tid : C0e + C_len + (tid - 32);
            if (e < (fast_pad ? A_pad : C0e + C_pad)) {
                const float f = fast_pad ? SORTED_FAR : 0.f;
                C0[e] = make_float4(f, f, f, f);
                C1[e] = make_float4(f, f, 0.f, 0.f);
                if (!FORCE) C2[e] = make_float4(0.f, 0.f, 0.f, 0.f);
                C3[e] = make_float2(0.f, 0.f);
                CI[e] = -1;
                CJ[e] = -1;
                CM[e] = 0;
            }
        }

        // ---- i state, two i's per packed register: k = 2 kp (.x) and 2 kp + 1 (.y) ----
        float2 xi[KP], yi[KP], zi[KP], ki[KP], wi[KP];
        float2 fxi[KP], fyi[KP], fzi[KP];
        float2 ax[KP], ay[KP], az[KP];
        float hx[IPT], hy[IPT], hz[IPT], lx[IPT], ly[IPT], lz[IPT];
#pragma unroll
        for (int kp = 0; kp < KP; ++kp) {
            const int ia = v.p0 + I * B + (2 * kp) * SYM_T + tid, ib = ia + SYM_T;
            const float4 a0 = a.s.p0[ia], b0 = a.s.p0[ib], a1 = a.s.p1[ia], b1 = a.s.p1[ib];
            xi[kp] = make_float2(-a0.x, -b0.x);
            yi[kp] = make_float2(-a0.z, -b0.z);
            zi[kp] = make_float2(-a1.x, -b1.x);
            if (FORCE) {
                wi[kp] = make_float2(a1.z, b1.z);
                ki[kp] = make_float2(a.s.k2[ia].x, a.s.k2[ib].x);
            } else {
                ki[kp] = make_float2(a1.z, b1.z);
                const float4 fa = a.s.q0[ia], fb = a.s.q0[ib];
                fxi[kp] = make_float2(fa.x, fb.x);
                fyi[kp] = make_float2(fa.z, fb.z);
                fzi[kp] = make_float2(a.s.q1[ia].x, a.s.q1[ib].x);
            }
            ax[kp] = ay[kp] = az[kp] = make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            hx[k] = hy[k] = hz[k] = lx[k] = ly[k] = lz[k] = 0.f;
            const int il = I * B + k * SYM_T + tid;
            IP[k * SYM_T + tid] = il < v.n ? a.perm[v.o0 + il] : -1;  // for the near pairs
        }
        __syncthreads();  // the lists are complete (and wcnt may be rewritten by the next item)

        const int nfs = A_pad >> 5, nms = B_used >> 5, nsub = nfs + nms + (C_pad >> 5);
        // j-side partials of the item, interleaved per droplet: [j][warp][3] (the reduction adds the warps in order)
        double *PJ = a.s.pj + (size_t)q * NW * 3 * plane + warp * 3;
        {
            for (int sub = 0; sub < nsub; ++sub) {
                float2 sx = make_float2(0.f, 0.f), sy = sx, sz = sx;
                bool had_exact = false;
#define DEM_SORTED_SUBTILE(MODE, MASK)                                                                            \
    sorted_subtile<IPT, PER, FORCE, MODE, MASK>(a, C0, C1, C2, C3, CI, CJ, IP, 32 * sub, lane, warp, diag, v,     \
                                                inv_ell, fscale_inv, invL2, magic2, nmagic2, nL2, hm, xi, yi, zi, ki, \
                                                wi, fxi, fyi, fzi, ax, ay, az, hx, hy, hz, lx, ly, lz, jnear, nq, PJ, \
                                                sx, sy, sz, had_exact)
                if (sub < nfs) {
                    DEM_SORTED_SUBTILE(MODE_FAST, 0);
                } else if (sub < nfs + nms) {
                    const int mask = __reduce_or_sync(0xffffffffu, (unsigned)CM[32 * sub + lane]);  // same in every warp
                    switch (mask) {
                        case 1: DEM_SORTED_SUBTILE(MODE_MASKED, 1); break;
                        case 2: DEM_SORTED_SUBTILE(MODE_MASKED, 2); break;
                        case 3: DEM_SORTED_SUBTILE(MODE_MASKED, 3); break;
                        case 4: DEM_SORTED_SUBTILE(MODE_MASKED, 4); break;
                        case 5: DEM_SORTED_SUBTILE(MODE_MASKED, 5); break;
                        case 6: DEM_SORTED_SUBTILE(MODE_MASKED, 6); break;
                        default: DEM_SORTED_SUBTILE(MODE_MASKED, 7); break;
                    }
                } else {
                    DEM_SORTED_SUBTILE(MODE_SLOW, 7);
                }
#undef DEM_SORTED_SUBTILE
                if (!diag) {  // the sums are back with the lanes owning their list entries
                    double vx = (double)(sx.x + sx.y), vy = (double)(sy.x + sy.y), vz = (double)(sz.x + sz.y);
                    if (had_exact) {  // warp-uniform: this sub-tile left exact j-side terms in jnear
                        __syncwarp();
                        vx += jnear[warp][0][lane];
                        vy += jnear[warp][1][lane];
                        vz += jnear[warp][2][lane];
                        jnear[warp][0][lane] = jnear[warp][1][lane] = jnear[warp][2][lane] = 0.0;
                        __syncwarp();
                    }
                    const int jo = CI[32 * sub + lane];
                    if (jo >= 0) {
                        double *d = PJ + (size_t)jo * NW * 3;
                        d[0] = vx;
                        d[1] = vy;
                        d[2] = vz;
                    }
                }
                if ((sub & 1) || sub == nsub - 1) {  // fold the FP32 i-side runs every 64 j and at the end
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
        __syncwarp();
        if (nq_count[warp] != 0)  // the pairs still queued (their j entries' partial sums are written)
            near_flush<IPT, PER, FORCE>(a, CI, CJ, IP, lane, warp, diag, v, inv_ell, fscale_inv, -1, nq, jnear, PJ,
                                        hx, hy, hz, lx, ly, lz);
        __syncthreads();  // every warp is done with the lists before the next item rebuilds them
        double *PI = a.s.pi + (size_t)q * 3 * plane;  // interleaved per droplet: [i][3]
        const double sg = FORCE ? -1.0 : 1.0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int li = k * SYM_T + tid;
            PI[3 * li] = sg * ((double)hx[k] + (double)lx[k]);
            PI[3 * li + 1] = sg * ((double)hy[k] + (double)ly[k]);
            PI[3 * li + 2] = sg * ((double)hz[k] + (double)lz[k]);
        }
    }
}

// Per block of the packed layout: the bins of its stored coordinates that hold a droplet, per axis.
__global__ void sorted_occupancy_kernel(const SymBoxes t, int B, const float4 *__restrict__ p0,
                                        const float4 *__restrict__ p1, uint32_t *__restrict__ occ) {
    double L = t.L1;
    const unsigned long long *scales = t.scales1;
    if (t.nbox > 1) {
        const int b = box_index(t.poff, t.nbox, (int)blockIdx.x * B);
        L = t.L[b];
        scales = t.scales + 2 * b;
    }
    const double inv_ell = pow2_inv_of(scales[0]);
    const float Ls = (float)(L * inv_ell), invLs = (float)(1.0 / (L * inv_ell));
    uint32_t *o = occ + (size_t)blockIdx.x * 3 * AMB_WORDS;
    for (int l = threadIdx.x; l < B; l += blockDim.x) {
        const int p = blockIdx.x * B + l;
        const float4 A = p0[p], Bv = p1[p];
        const float v[3] = {A.x, A.z, Bv.x};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int b = amb_bin(v[c], Ls, invLs);
            atomicOr(&o[c * AMB_WORDS + (b >> 5)], 1u << (b & 31));
        }
    }
}

// Per block of the packed layout: bounds of the stored coordinates and the largest k r.
template <bool FORCE>
__global__ void __launch_bounds__(SYM_T) sorted_bounds_kernel(int B, const float4 *__restrict__ p0,
                                                              const float4 *__restrict__ p1,
                                                              const float2 *__restrict__ k2,
                                                              float4 *__restrict__ bounds) {
    __shared__ float red[7][SYM_T / 32];
    float mn[3] = {3.0e38f, 3.0e38f, 3.0e38f}, mx[3] = {-3.0e38f, -3.0e38f, -3.0e38f}, km = 0.f;
    for (int l = threadIdx.x; l < B; l += SYM_T) {
        const int p = blockIdx.x * B + l;
        const float4 A = p0[p], Bv = p1[p];
        const float v[3] = {A.x, A.z, Bv.x};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            mn[c] = fminf(mn[c], v[c]);
            mx[c] = fmaxf(mx[c], v[c]);
        }
        km = fmaxf(km, FORCE ? k2[p].x : Bv.z);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            mn[c] = fminf(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
            mx[c] = fmaxf(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
        }
        km = fmaxf(km, __shfl_xor_sync(0xffffffffu, km, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        for (int c = 0; c < 3; ++c) {
            red[c][w] = mn[c];
            red[3 + c][w] = mx[c];
        }
        red[6][w] = km;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int ww = 1; ww < SYM_T / 32; ++ww) {
            for (int c = 0; c < 3; ++c) {
                red[c][0] = fminf(red[c][0], red[c][ww]);
                red[3 + c][0] = fmaxf(red[3 + c][0], red[3 + c][ww]);
            }
            red[6][0] = fmaxf(red[6][0], red[6][ww]);
        }
        bounds[2 * blockIdx.x] = make_float4(red[0][0], red[1][0], red[2][0], red[6][0]);
        bounds[2 * blockIdx.x + 1] = make_float4(red[3][0], red[4][0], red[5][0], 0.f);
    }
}

// Packed, zero-padded layout of the symmetric passes (see SymArgs).
template <bool FORCE>
__global__ void prep_sym_kernel(const SymBoxes t, const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ z, const double *__restrict__ r,
                                const double *__restrict__ fx, const double *__restrict__ fy,
                                const double *__restrict__ fz, double k_near, const int32_t *__restrict__ perm,
                                float4 *__restrict__ p0, float4 *__restrict__ p1, float4 *__restrict__ q0,
                                float2 *__restrict__ k2q1) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < t.npad_total; p += gridDim.x * blockDim.x) {
        int o0 = 0, nb = t.n1, pb = 0;
        double L = t.L1;
        const unsigned long long *sc = t.scales1;
        if (t.nbox > 1) {
            const int b = box_index(t.poff, t.nbox, p);
            o0 = t.off[b];
            nb = t.off[b + 1] - o0;
            pb = t.poff[b];
            L = t.L[b];
            sc = t.scales + 2 * b;
        }
        const int l = p - pb;
        float X = 0.f, Y = 0.f, Z = 0.f, W = 0.f, K = 0.f, Fx = 0.f, Fy = 0.f, Fz = 0.f;
        if (l < nb) {
            const int i = perm ? perm[o0 + l] : o0 + l;  // perm: each box's droplets in Morton order
            const double s = pow2_inv_of(sc[0]);
            const double center = 0.5 * L;
            const double rs = r[i] * s;
            X = (float)((x[i] - center) * s);
            Y = (float)((y[i] - center) * s);
            Z = (float)((z[i] - center) * s);
            W = (float)(rs * rs * rs);
            K = (float)(k_near * rs);
            if (!FORCE) {
                const double q = pow2_inv_of(sc[1]);
                Fx = (float)(fx[i] * q);
                Fy = (float)(fy[i] * q);
                Fz = (float)(fz[i] * q);
            }
        }
        if (FORCE) {
            p0[p] = make_float4(X, X, Y, Y);
            p1[p] = make_float4(Z, Z, W, W);
            k2q1[p] = make_float2(K, K);
        } else {
            p0[p] = make_float4(-X, -X, -Y, -Y);
            p1[p] = make_float4(-Z, -Z, K, K);
            q0[p] = make_float4(Fx, Fx, Fy, Fy);
            k2q1[p] = make_float2(Fz, Fz);
        }
    }
}

// out_c[d] = factor_d * (sum over items (K, J>=K) of the i side + sum over items (I<K, K) of the j side)
// PLANAR (mixed_sym_kernel): partials as planes [item][3][B]; else (the sorted kernel) interleaved per droplet,
// i side [item][B][3] and j side [item][B][JW][3], so that a thread reads contiguous records.
// RED_SPLIT consecutive lanes share a droplet: lane q of the group adds the items q, q + RED_SPLIT, ... of both
// sides, and the groups' sums are combined by a fixed butterfly, so the order depends on K and nbk only.
constexpr int RED_SPLIT = 4;
// Build knobs of the reduction: 16-byte loads of the sorted kernel's j records, and the
// resident CTAs per SM its registers are budgeted for.
#ifndef DEM_RED_VEC
#define DEM_RED_VEC 1
#endif
#ifndef DEM_RED_MIN_CTAS
#define DEM_RED_MIN_CTAS 4
#endif

template <bool FORCE, int JW, bool PLANAR>
__global__ void __launch_bounds__(256, DEM_RED_MIN_CTAS) reduce_sym_kernel(const SymBoxes t, int B, const double *__restrict__ pi,
                                                         const double *__restrict__ pj, const double *__restrict__ r,
                                                         double coeff, double *__restrict__ ox,
                                                         double *__restrict__ oy, double *__restrict__ oz,
                                                         uint32_t *err, const int32_t *__restrict__ perm) {
    const size_t plane = (size_t)B;
    const int lane = threadIdx.x & 31, q = lane % RED_SPLIT;
    const int stride = gridDim.x * (blockDim.x / RED_SPLIT);
    // whole warps walk the droplets together (the butterfly below needs every lane)
    for (int d0 = (blockIdx.x * blockDim.x + threadIdx.x - lane) / RED_SPLIT; d0 < t.n_total; d0 += stride) {
        // d: position in the packed layout; with perm (one box in Morton order) its droplet is perm[d]
        const int d = d0 + lane / RED_SPLIT;
        const bool live = d < t.n_total;
        double sx = 0.0, sy = 0.0, sz = 0.0;
        int o0 = 0, nbk = t.npad1 / B, ib = 0;
        const unsigned long long *sc = t.scales1;
        if (live) {
            if (t.nbox > 1) {
                const int b = box_index(t.off, t.nbox, d);
                o0 = t.off[b];
                nbk = (t.poff[b + 1] - t.poff[b]) / B;
                ib = t.ioff[b];
                sc = t.scales + 2 * b;
            }
            const int l = d - o0;
            const int K = l / B, lb = l - K * B;
            // i side: items (K, K + q), (K, K + q + RED_SPLIT), ...
            {
                const double *P =
                    pi + (size_t)(ib + rows_before(K, nbk) + q) * 3 * plane + (PLANAR ? lb : 3 * lb);
                const size_t step = RED_SPLIT * 3 * plane, cs = PLANAR ? plane : 1;
#pragma unroll 4
                for (int Jb = K + q; Jb < nbk; Jb += RED_SPLIT, P += step) {
                    const double a = P[0], b = P[cs], c = P[2 * cs];
                    sx += a;
                    sy += b;
                    sz += c;
                }
            }
            // j side: items (q, K), (q + RED_SPLIT, K), ...; item (Ib, K) = rows_before(Ib) + K - Ib; an item
            // holds JW sets of j-side partials (one per warp of the sorted kernel), added in order
            {
                const size_t wstep = 3 * plane;
                const size_t off = PLANAR ? (size_t)lb : (size_t)lb * JW * 3;
#pragma unroll 2
                for (int Ib = q; Ib < K; Ib += RED_SPLIT) {
                    const long long item = ib + rows_before(Ib, nbk) + K - Ib;
                    const double *P = pj + (size_t)item * JW * wstep + off;
                    double a[JW], b[JW], c[JW];
                    if (DEM_RED_VEC && !PLANAR && JW % 2 == 0) {  // JW x 3 doubles, 16-byte aligned: vector loads
                        const double2 *P2 = reinterpret_cast<const double2 *>(P);
                        double rec[3 * JW];
#pragma unroll
                        for (int h = 0; h < 3 * JW / 2; ++h) {
                            const double2 v2 = P2[h];
                            rec[2 * h] = v2.x;
                            rec[2 * h + 1] = v2.y;
                        }
#pragma unroll
                        for (int w = 0; w < JW; ++w) {
                            a[w] = rec[3 * w];
                            b[w] = rec[3 * w + 1];
                            c[w] = rec[3 * w + 2];
                        }
                    } else {
#pragma unroll
                        for (int w = 0; w < JW; ++w) {
                            if (PLANAR) {
                                a[w] = P[w * wstep];
                                b[w] = P[w * wstep + plane];
                                c[w] = P[w * wstep + 2 * plane];
                            } else {
                                a[w] = P[3 * w];
                                b[w] = P[3 * w + 1];
                                c[w] = P[3 * w + 2];
                            }
                        }
                    }
#pragma unroll
                    for (int w = 0; w < JW; ++w) {
                        sx += a[w];
                        sy += b[w];
                        sz += c[w];
                    }
                }
            }
        }
        // (s0 + s1) + (s2 + s3) on every lane of the group: each add sees the same two operands in either order
#pragma unroll
        for (int o = 1; o < RED_SPLIT; o <<= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
            sz += __shfl_xor_sync(0xffffffffu, sz, o);
        }
        if (!live || q != 0) continue;
        const double s = pow2_inv_of(sc[0]);
        const int od = perm ? perm[d] : d;
        double f;
        if (FORCE) {
            const double ell = 1.0 / s;
            const double rs = r[od] * s;
            f = coeff * ipow3(rs) * ell * ell;
        } else {
            f = coeff * s / pow2_inv_of(sc[1]);
        }
        const double vx = f * sx, vy = f * sy, vz = f * sz;
        if (!(isfinite(vx) && isfinite(vy) && isfinite(vz))) raise_device_error(err, DEM_DEVERR_NONFINITE);
        ox[od] = vx;
        oy[od] = vy;
        oz[od] = vz;
    }
}

// Per-box max |v| (as the bit pattern of a non-negative double).
__global__ void maxabs_boxes_kernel(const SymBoxes t, const double *__restrict__ a, const double *__restrict__ b,
                                    const double *__restrict__ c, unsigned long long *__restrict__ scales, int slot) {
    for (int base = blockIdx.x * blockDim.x; base < t.n_total; base += gridDim.x * blockDim.x) {
        const int d = base + threadIdx.x;
        double m = 0.0;
        int box = -1;
        if (d < t.n_total) {
            box = box_index(t.off, t.nbox, d);
            m = fabs(a[d]);
            if (b) m = fmax(m, fabs(b[d]));
            if (c) m = fmax(m, fabs(c[d]));
        }
        const int box0 = __shfl_sync(0xffffffffu, box, 0);
        if (__all_sync(0xffffffffu, box == box0 || box < 0)) {  // one box in this warp: one atomic
#pragma unroll
            for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0 && box0 >= 0 && m > 0.0)
                atomicMax(&scales[2 * box0 + slot], (unsigned long long)__double_as_longlong(m));
        } else if (box >= 0 && m > 0.0) {
            atomicMax(&scales[2 * box + slot], (unsigned long long)__double_as_longlong(m));
        }
    }
}

int launch_maxabs_boxes(dem_ctx *ctx, const SymBoxes &t, const double *a, const double *b, const double *c,
                        unsigned long long *scales, int slot, cudaStream_t s) {
    const int grid = max(1, min(ceil_div(t.n_total, 256), 4 * ctx->sm_count));
    maxabs_boxes_kernel<<<grid, 256, 0, counted(s)>>>(t, a, b, c, scales, slot);
    return dem_check_launch(ctx, "maxabs (boxes)");
}

template <int IPT, bool FORCE>
static const void *sym_kernel_ptr(bool per) {
    return per ? (const void *)mixed_sym_kernel<IPT, true, FORCE> : (const void *)mixed_sym_kernel<IPT, false, FORCE>;
}

int sym_resident_ctas(int ipt, bool per, bool force) {
    const void *f = ipt >= 4 ? (force ? sym_kernel_ptr<4, true>(per) : sym_kernel_ptr<4, false>(per))
                             : (force ? sym_kernel_ptr<2, true>(per) : sym_kernel_ptr<2, false>(per));
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, SYM_T, 0) != cudaSuccess) occ = 1;
    return occ > 0 ? occ : 1;
}

template <int IPT, bool FORCE>
static void launch_sym(bool per, const SymArgs &a, int grid, cudaStream_t s) {
    if (per)
        mixed_sym_kernel<IPT, true, FORCE><<<grid, SYM_T, 0, counted(s)>>>(a);
    else
        mixed_sym_kernel<IPT, false, FORCE><<<grid, SYM_T, 0, counted(s)>>>(a);
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

size_t sym_workspace_bytes(long long npad_total, long long items_total, int B) {
    return align256((size_t)npad_total * 64) + (size_t)(2 * items_total * 3 * (long long)B) * sizeof(double);
}

// Workspace bytes of the symmetric schedule for one box of n droplets: the
// packed layout and partial sums, plus the Morton order and the per-block
// bounds of the sorted kernel.
size_t sym_sorted_extra_bytes(long long n_total, long long npad_total, long long items_total, int B) {
    const long long nb = npad_total / B;
    // (SYM_T / 32 - 1) more j-side planes per item than the plain kernel's, then the order, bounds and bitmaps
    return (size_t)((SYM_T / 32 - 1) * items_total * 3 * (long long)B) * sizeof(double) +
           align256(morton_ws_bytes(n_total > 0 ? (int)n_total : 1)) + align256((size_t)nb * 2 * sizeof(float4)) +
           (size_t)nb * 3 * AMB_WORDS * sizeof(uint32_t);
}

size_t sym_partial_bytes(int n, int ipt) {
    const long long B = (long long)SYM_T * ipt;
    const long long nb = (n + B - 1) / B;
    return sym_workspace_bytes(nb * B, nb * (nb + 1) / 2, (int)B) +
           sym_sorted_extra_bytes(n, nb * B, nb * (nb + 1) / 2, (int)B);
}

// 30-bit Morton key of each droplet's cell in its box's cube [0, L_b)^3 (1024
// cells per axis, clamped), the same expression for one box and for every box
// of an ensemble, so that a box sorts into the same order either way.
__global__ void box_morton_keys_kernel(const SymBoxes t, const double *__restrict__ x, const double *__restrict__ y,
                                       const double *__restrict__ z, uint32_t *__restrict__ keys,
                                       int32_t *__restrict__ idx) {
    auto spread10 = [](uint32_t v) {  // bit k -> bit 3k
        v &= 0x3ffu;
        v = (v | (v << 16)) & 0x030000FFu;
        v = (v | (v << 8)) & 0x0300F00Fu;
        v = (v | (v << 4)) & 0x030C30C3u;
        v = (v | (v << 2)) & 0x09249249u;
        return v;
    };
    auto cell10 = [](double p, double inv) {
        const int c = (int)floor(p * inv * 1024.0);
        return (uint32_t)(c < 0 ? 0 : (c > 1023 ? 1023 : c));
    };
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < t.n_total; d += gridDim.x * blockDim.x) {
        const double inv = 1.0 / (t.nbox > 1 ? t.L[box_index(t.off, t.nbox, d)] : t.L1);
        keys[d] = (spread10(cell10(x[d], inv)) << 2) | (spread10(cell10(y[d], inv)) << 1) | spread10(cell10(z[d], inv));
        idx[d] = d;
    }
}

// keys[k] = the box of droplet idx[k] (the last, most significant sort digit of an ensemble).
__global__ void box_of_kernel(const SymBoxes t, const int32_t *__restrict__ idx, uint32_t *__restrict__ keys) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < t.n_total; k += gridDim.x * blockDim.x)
        keys[k] = (uint32_t)box_index(t.off, t.nbox, idx[k]);
}

template <int IPT, bool PER, bool FORCE>
static cudaError_t sorted_attr() {
    return cudaFuncSetAttribute(mixed_sym_sorted_kernel<IPT, PER, FORCE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                sorted_smem_bytes<IPT, FORCE>());
}

// Raises the dynamic shared-memory limit of every sorted pair kernel on the
// context's (current) device.  Called when a context is created, so that no
// pass has to do it (possibly inside a stream capture).
int sym_sorted_prepare(dem_ctx *ctx) {
    const cudaError_t es[] = {sorted_attr<4, true, true>(),  sorted_attr<4, true, false>(),
                              sorted_attr<4, false, true>(), sorted_attr<4, false, false>(),
                              sorted_attr<2, true, true>(),  sorted_attr<2, true, false>(),
                              sorted_attr<2, false, true>(), sorted_attr<2, false, false>()};
    for (cudaError_t e : es)
        if (e != cudaSuccess) return dem_check_cuda(ctx, e, "sorted pass: shared memory attribute");
    return DEM_OK;
}

template <int IPT, bool PER, bool FORCE>
static int launch_sorted(dem_ctx *ctx, const SortedArgs &a, int grid, cudaStream_t s) {
    mixed_sym_sorted_kernel<IPT, PER, FORCE><<<grid, SYM_T, sorted_smem_bytes<IPT, FORCE>(), counted(s)>>>(a);
    return DEM_OK;
}

// Droplets of every box in Morton order: sort, pack, per-block bounds, the pair
// kernel with fast, medium and slow lists, then the fixed-order reduction
// through the permutation.  ctas = 0: one CTA per block pair, else a
// persistent grid of that many.  At most 256 boxes (the key's box field).
template <bool FORCE>
static int run_sym_sorted(dem_ctx *ctx, const SymBoxes &t, int ipt, int ctas, bool per, const MixedArgs &m,
                          double *work, double coeff, double *ox, double *oy, double *oz, cudaStream_t s) {
    const int B = SYM_T * ipt;
    const int n = t.n_total;
    const int nb = t.npad_total / B;
    if (n == 0) return DEM_OK;
    char *base = reinterpret_cast<char *>(work);
    const size_t np = (size_t)t.npad_total;
    float4 *p0 = reinterpret_cast<float4 *>(base);
    float4 *p1 = p0 + np;
    float4 *q0 = p1 + np;
    float2 *k2q1 = reinterpret_cast<float2 *>(q0 + np);
    double *pi = reinterpret_cast<double *>(base + align256(np * 64));
    double *pj = pi + (size_t)t.items_total * 3 * B;  // [items][SYM_T / 32][3][B]
    char *extra = base + sym_workspace_bytes(t.npad_total, t.items_total, B) +
                  (size_t)((SYM_T / 32 - 1) * (long long)t.items_total * 3 * B) * sizeof(double);
    const MortonWs mw = morton_ws_carve(extra, n);
    float4 *bounds = reinterpret_cast<float4 *>(extra + align256(morton_ws_bytes(n)));
    uint32_t *occ = reinterpret_cast<uint32_t *>(extra + align256(morton_ws_bytes(n)) +
                                                 align256((size_t)nb * 2 * sizeof(float4)));
    // sorted position -> droplet; box b keeps positions [off[b], off[b + 1]).  An open single box
    // sorts in its droplets' bounding cube; boxes of an ensemble and periodic boxes in [0, L_b)^3,
    // then (ensembles) a stable pass on the box index groups every box's droplets
    int rc = DEM_OK;
    const int32_t *perm = t.nbox > 1 ? mw.idx[1] : mw.idx[0];
    const int kg = max(1, min(ceil_div(n, 256), 8 * ctx->sm_count));
    auto &ord = ctx->sym_order;
    const bool reuse = ctx->sym_reuse_order && ord.work == work && ord.n_total == n &&
                       ord.npad_total == t.npad_total && ord.nbox == t.nbox && ord.ipt == ipt && ord.per == (int)per;
    if (!reuse) {  // (reuse: the caller's previous pass sorted these positions into this workspace)
        ord.work = nullptr;
        if (t.nbox == 1 && !per) {
            rc = morton_order(ctx, n, m.x, m.y, m.z, 0, m.L, mw, s);
        } else {
            box_morton_keys_kernel<<<kg, 256, 0, counted(s)>>>(t, m.x, m.y, m.z, mw.keys[0], mw.idx[0]);
            rc = radix_sort_pairs(ctx, n, mw, s);
            if (!rc && t.nbox > 1) {
                box_of_kernel<<<kg, 256, 0, counted(s)>>>(t, mw.idx[0], mw.keys[0]);
                rc = radix_pass(ctx, n, mw.keys[0], mw.idx[0], mw.keys[1], mw.idx[1], 0, mw.hist, s);
            }
        }
        if (rc) return rc;
        ord.work = work;
        ord.n_total = n;
        ord.npad_total = t.npad_total;
        ord.nbox = t.nbox;
        ord.ipt = ipt;
        ord.per = (int)per;
    }
    const int pgrid = max(1, min(ceil_div(t.npad_total, 256), 4 * ctx->sm_count));
    prep_sym_kernel<FORCE><<<pgrid, 256, 0, counted(s)>>>(t, m.x, m.y, m.z, m.r, m.fx, m.fy, m.fz,
                                                          FORCE ? ctx->tuning.near_force : ctx->tuning.near_oseen,
                                                          perm, p0, p1, q0, k2q1);
    sorted_bounds_kernel<FORCE><<<nb, SYM_T, 0, counted(s)>>>(B, p0, p1, k2q1, bounds);
    if (per) {
        rc = dem_check_cuda(ctx, cudaMemsetAsync(occ, 0, (size_t)nb * 3 * AMB_WORDS * sizeof(uint32_t), s), "memset");
        if (rc) return rc;
        sorted_occupancy_kernel<<<nb, SYM_T, 0, counted(s)>>>(t, B, p0, p1, occ);
    }
    rc = dem_check_launch(ctx, "sorted pass prep");
    if (rc) return rc;
    SortedArgs a;
    a.s.t = t;
    a.s.p0 = p0;
    a.s.p1 = p1;
    a.s.q0 = q0;
    a.s.k2 = k2q1;
    a.s.q1 = k2q1;
    a.s.m = m;
    a.s.pi = pi;
    a.s.pj = pj;
    a.perm = perm;
    a.bounds = bounds;
    a.occ = occ;
    const int grid = ctas > 0 ? min(ctas, t.items_total) : t.items_total;
    dem_prof_begin(ctx, FORCE ? "mixed_force_pass" : "mixed_convection_pass", s);
    if (ipt == 4)
        rc = per ? launch_sorted<4, true, FORCE>(ctx, a, grid, s) : launch_sorted<4, false, FORCE>(ctx, a, grid, s);
    else
        rc = per ? launch_sorted<2, true, FORCE>(ctx, a, grid, s) : launch_sorted<2, false, FORCE>(ctx, a, grid, s);
    dem_prof_end(ctx, s);
    if (rc) return rc;
    rc = dem_check_launch(ctx, FORCE ? "mixed force (symmetric, Morton order)" : "mixed convection (symmetric, Morton order)");
    if (rc) return rc;
    const int rgrid = max(1, min(ceil_div(n, 256 / RED_SPLIT), 8 * ctx->sm_count));
    reduce_sym_kernel<FORCE, SYM_T / 32, false><<<rgrid, 256, 0, counted(s)>>>(t, B, pi, pj, m.r, coeff, ox, oy, oz,
                                                                               m.err, perm);
    return dem_check_launch(ctx, "mixed reduce (symmetric, Morton order)");
}

// Blocks in the caller's droplet order (DEM_SCHED_SYMMETRIC_PLAIN): every pair
// takes the minimum image and the tests in mixed_sym_kernel.
template <bool FORCE>
static int run_sym_plain(dem_ctx *ctx, const SymBoxes &t, int ipt, int ctas, bool per, const MixedArgs &m,
                         double *work, double coeff, double *ox, double *oy, double *oz, cudaStream_t s) {
    const int B = SYM_T * ipt;
    char *base = reinterpret_cast<char *>(work);
    const size_t np = (size_t)t.npad_total;
    float4 *p0 = reinterpret_cast<float4 *>(base);
    float4 *p1 = p0 + np;
    float4 *q0 = p1 + np;
    float2 *k2q1 = reinterpret_cast<float2 *>(q0 + np);
    const int pgrid = max(1, min(ceil_div(t.npad_total, 256), 4 * ctx->sm_count));
    prep_sym_kernel<FORCE><<<pgrid, 256, 0, counted(s)>>>(t, m.x, m.y, m.z, m.r, m.fx, m.fy, m.fz,
                                                          FORCE ? ctx->tuning.near_force : ctx->tuning.near_oseen,
                                                          nullptr, p0, p1, q0, k2q1);
    SymArgs a;
    a.t = t;
    a.p0 = p0;
    a.p1 = p1;
    a.q0 = q0;
    a.k2 = k2q1;
    a.q1 = k2q1;
    a.m = m;
    a.pi = reinterpret_cast<double *>(base + align256(np * 64));
    a.pj = a.pi + (size_t)t.items_total * 3 * B;
    const int grid = ctas > 0 ? min(ctas, t.items_total) : t.items_total;
    dem_prof_begin(ctx, FORCE ? "mixed_force_pass" : "mixed_convection_pass", s);
    if (ipt == 4)
        launch_sym<4, FORCE>(per, a, grid, s);
    else
        launch_sym<2, FORCE>(per, a, grid, s);
    dem_prof_end(ctx, s);
    int rc = dem_check_launch(ctx, FORCE ? "mixed force (symmetric)" : "mixed convection (symmetric)");
    if (rc) return rc;
    const int rgrid = max(1, min(ceil_div(t.n_total, 256 / RED_SPLIT), 8 * ctx->sm_count));
    reduce_sym_kernel<FORCE, 1, true><<<rgrid, 256, 0, counted(s)>>>(t, B, a.pi, a.pj, m.r, coeff, ox, oy, oz, m.err,
                                                                     nullptr);
    return dem_check_launch(ctx, "mixed reduce (symmetric)");
}

template <bool FORCE>
int run_sym_boxes(dem_ctx *ctx, const SymBoxes &t, int ipt, int ctas, bool per, const MixedArgs &m, double *work,
                  double coeff, double *ox, double *oy, double *oz, cudaStream_t s) {
    ipt = ipt >= 4 ? 4 : 2;
    if (t.n_total == 0) return DEM_OK;
    if (ctx->tuning.schedule == DEM_SCHED_SYMMETRIC_PLAIN || t.nbox > 256)
        return run_sym_plain<FORCE>(ctx, t, ipt, ctas, per, m, work, coeff, ox, oy, oz, s);
    return run_sym_sorted<FORCE>(ctx, t, ipt, ctas, per, m, work, coeff, ox, oy, oz, s);
}

template int run_sym_boxes<true>(dem_ctx *, const SymBoxes &, int, int, bool, const MixedArgs &, double *, double,
                                 double *, double *, double *, cudaStream_t);
template int run_sym_boxes<false>(dem_ctx *, const SymBoxes &, int, int, bool, const MixedArgs &, double *, double,
                                  double *, double *, double *, cudaStream_t);

// One box (the library's single-system calls): the table lives in kernel arguments.
template <bool FORCE>
int run_sym_pass(dem_ctx *ctx, int n, int ipt, bool per, const MixedArgs &m, double *work, const double *r,
                 double coeff, double *ox, double *oy, double *oz, cudaStream_t s) {
    ipt = ipt >= 4 ? 4 : 2;
    const long long B = (long long)SYM_T * ipt;
    const long long nb = (n + B - 1) / B;
    const long long items = nb * (nb + 1) / 2;
    if (items > 0x7fffffffLL || nb * B > 0x7fffffffLL)
        return dem_set_error(ctx, DEM_E_CAPACITY, "symmetric schedule: too many blocks");
    SymBoxes t{};
    t.nbox = 1;
    t.n_total = t.n1 = n;
    t.npad_total = t.npad1 = (int)(nb * B);
    t.items_total = (int)items;
    t.L1 = m.L;
    t.scales1 = m.scales;
    MixedArgs mm = m;
    mm.r = r;
    return run_sym_boxes<FORCE>(ctx, t, ipt, 0, per, mm, work, coeff, ox, oy, oz, s);
}

template int run_sym_pass<true>(dem_ctx *, int, int, bool, const MixedArgs &, double *, const double *, double,
                                double *, double *, double *, cudaStream_t);
template int run_sym_pass<false>(dem_ctx *, int, int, bool, const MixedArgs &, double *, const double *, double,
                                 double *, double *, double *, cudaStream_t);

}  // namespace dem
