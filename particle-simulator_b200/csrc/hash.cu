// hash.cu -- spatial-hash collision detection with the reference's exact
// cell, hash and distance semantics, producing the sorted unique pair set.
//
// dem/collision_detector/spatial_hash_collision_detector.py:
//   _hash_cell :74-76, _assign_cells :79-112, _prefix_sum :115-123,
//   _scatter_particles :126-132, _detect_collisions :135-229, detect :233-316.
//
// Pipeline (all on the device, no host synchronisation):
//   1. max radius            -> cell = 2 max r, grid = max(1, ceil(L / cell))
//   2. bucket of every droplet, bucket counts (atomics)
//   3. exclusive scan of the counts (bucket starts), scatter into buckets
//   4. per droplet i: the distinct hash buckets of its 27 neighbour cells; count
//      the j > i in them with MIC distance <= r_i + r_j (threads take the
//      droplets in bucket order, so the lanes of a warp share candidate lists)
//   5. exclusive scan of the per-i counts -> pair offsets (lexicographic order)
//   6. per droplet i: write its pairs, sort its j's ascending
// Memory roofline: the chain is bounded by HBM and latency, not arithmetic.  Its
// algorithmic bytes per detection are 48 N + 8 T + 8 K (N droplets, T table
// slots, K pairs): position and radius read once (32 B), bucket id and bucket
// slot written and read (16 B), bucket starts written and read (8 B per slot),
// 8 B per pair written.
// The candidate set of a droplet is exactly the reference's (the same buckets,
// including buckets shared by aliased cells), and the distance test is the
// same IEEE expression (this file is compiled with -fmad=false), so the pair
// set is bit-identical to the reference's np.unique output.
#include "common.cuh"
#include "scan.cuh"

namespace dem {

struct HashParams {
    double cell;
    int32_t grid;
    int32_t valid;
};

__device__ __forceinline__ unsigned long long ordered_bits(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered_bits(unsigned long long o) {
    const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    return __longlong_as_double((long long)b);
}

__global__ void max_kernel(int n, const double *__restrict__ r, unsigned long long *__restrict__ slot) {
    unsigned long long m = 0ull;  // below every ordered value
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long o = ordered_bits(r[i]);
        m = o > m ? o : m;
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, m, off);
        m = t > m ? t : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(slot, m);
}

// even_cells = 0: the reference's grid, cell = 2 max r and grid = ceil(L / cell)
// (a periodic box whose side is not a whole number of cells gets a partial last
// cell, across which touching pairs one cell apart are not compared -- the
// reference's pair set, kept bit-exact).  even_cells = 1 (the generator's own
// use): grid = floor(L / (2 max r)) whole cells of side L / grid >= 2 max r, so
// every touching pair is compared across the periodic faces too.
__global__ void hash_params_kernel(const unsigned long long *__restrict__ slot, double L, int even_cells,
                                   HashParams *__restrict__ hp) {
    const double max_radius = from_ordered_bits(*slot);
    double cell = 2.0 * max_radius;  // :258
    HashParams p;
    p.valid = cell > 0 ? 1 : 0;  // :259-260
    double g = p.valid ? (even_cells ? floor(L / cell) : ceil(L / cell)) : 1.0;
    if (!(g >= 1.0)) g = 1.0;
    if (g > 1073741824.0) g = 1073741824.0;
    if (even_cells && p.valid) cell = L / g;
    p.cell = cell;
    p.grid = (int32_t)g;  // :262
    *hp = p;
}

__device__ __forceinline__ int32_t hash_cell(int32_t ix, int32_t iy, int32_t iz, int32_t mask) {
    const uint32_t h = ((uint32_t)ix * 73856093u) ^ ((uint32_t)iy * 19349663u) ^ ((uint32_t)iz * 83492791u);
    return (int32_t)(h & (uint32_t)mask);
}

__device__ __forceinline__ int32_t floor_mod(int32_t a, int32_t m) {
    const int32_t q = a % m;
    return q < 0 ? q + m : q;
}

// floor_mod(a, m) for a in [-1, m] (a neighbour of a periodic cell coordinate)
__device__ __forceinline__ int32_t wrap1(int32_t a, int32_t m) {
    a += a < 0 ? m : 0;
    return a >= m ? a - m : a;
}

__device__ __forceinline__ int32_t cell_coord(double p, double cell, int32_t grid, bool periodic) {
    int32_t v = (int32_t)floor(p / cell);
    if (periodic) return floor_mod(v, grid);
    return v < 0 ? 0 : (v >= grid ? grid - 1 : v);
}

__global__ void assign_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const HashParams *__restrict__ hp, int periodic,
                              int32_t mask, int32_t *__restrict__ cell_hash, int32_t *__restrict__ bucket_count,
                              int32_t *__restrict__ cell_xyz) {
    const HashParams p = *hp;
    if (!p.valid) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t ix = cell_coord(x[i], p.cell, p.grid, periodic);
        const int32_t iy = cell_coord(y[i], p.cell, p.grid, periodic);
        const int32_t iz = cell_coord(z[i], p.cell, p.grid, periodic);
        const int32_t h = hash_cell(ix, iy, iz, mask);
        cell_hash[i] = h;
        if (cell_xyz) {  // [3][n], for the count pass
            cell_xyz[i] = ix;
            cell_xyz[n + i] = iy;
            cell_xyz[2 * (size_t)n + i] = iz;
        }
        atomicAdd(&bucket_count[h], 1);
    }
}

__global__ void scatter_kernel(int n, const int32_t *__restrict__ cell_hash, const HashParams *__restrict__ hp,
                               int32_t *__restrict__ cursor, int32_t *__restrict__ sorted_idx) {
    if (!hp->valid) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t slot = atomicAdd(&cursor[cell_hash[i]], 1);
        sorted_idx[slot] = i;
    }
}

// The reference's contact test sqrt(d2) <= s (s = r_i + r_j, the root correctly
// rounded), decided from d2 alone unless d2 lies within a relative 2^-45 of s^2.
// With s2 = RN(s * s): d2 > s2 (1 + 2^-45) implies sqrt(d2) > s (1 + 2^-47), above
// s + ulp(s) / 2, so the rounded root exceeds s; d2 <= s2 (1 - 2^-45) implies
// d2 < s^2, so the rounded root is <= s.  Both need s > 0 and s2 normal and
// finite (the relative bounds), else, and inside the band, the square root decides.
__device__ __forceinline__ bool contact_rn(double d2, double s) {
    const double s2 = s * s;
    const bool normal = s > 0.0 && s2 >= 0x1p-960 && s2 <= 0x1p+960;
    if (normal && d2 > s2 * (1.0 + 0x1p-45)) return false;
    if (normal && d2 <= s2 * (1.0 - 0x1p-45)) return true;
    return sqrt(d2) <= s;
}

// Visits every candidate j > i of droplet i (the distinct buckets of its 27
// neighbour cells) and calls f(j, multiplicity) for those in contact.
// PACKED: the droplets' (x, y), (z, r) in bucket order are in P (two double2
// per bucket slot, slot ti holding droplet i), so a bucket's candidates are
// read as contiguous 32-byte records instead of four scattered gathers, and
// their FP32 roundings in P32 reject the clearly separated candidates first.
// That test only drops a candidate whose FP32 distance exceeds the contact
// distance by far more than FP32 rounding can account for (a margin of
// 2^-17 (max |x_i| + L) plus 2^-18 of the radii sum; the per-axis distance is
// bounded below by the smaller of |d| and ||d| - L|, which covers either image
// the FP64 test may take); NaNs and overflowed bounds fail the comparison and
// go to the FP64 test, and a margin below 2^-100 turns the far test off.  So
// every pair the FP64 test accepts is still found.
template <bool PACKED, typename F>
__device__ __forceinline__ void for_each_contact(int i, int ti, const double *__restrict__ x,
                                                 const double *__restrict__ y, const double *__restrict__ z,
                                                 const double *__restrict__ r, const double2 *__restrict__ P,
                                                 const float4 *__restrict__ P32,
                                                 const HashParams &p, int periodic, double L, double halfL,
                                                 int32_t mask, int n, const int32_t *__restrict__ bstart,
                                                 const int32_t *__restrict__ sorted_idx, F &&f) {
    double xi, yi, zi, ri;
    if (PACKED) {
        const double2 a = P[2 * ti], b = P[2 * ti + 1];
        xi = a.x;
        yi = a.y;
        zi = b.x;
        ri = b.y;
    } else {
        xi = x[i];
        yi = y[i];
        zi = z[i];
        ri = r[i];
    }
    const int32_t cx = cell_coord(xi, p.cell, p.grid, periodic);
    const int32_t cy = cell_coord(yi, p.cell, p.grid, periodic);
    const int32_t cz = cell_coord(zi, p.cell, p.grid, periodic);
    float4 qi = make_float4(0.f, 0.f, 0.f, 0.f);
    float Lf = 0.f, marg = 0.f;
    if (PACKED) {
        qi = P32[ti];
        Lf = (float)L;
        marg = (float)(0x1p-17 * (fmax(fabs(xi), fmax(fabs(yi), fabs(zi))) + fabs(L)));
        qi.w = qi.w * (1.f + 0x1p-18f) + marg;  // r_i, widened: the far test adds r_j (1 + 2^-18)
        if (!(marg >= 0x1p-100f)) qi.w = INFINITY;  // coordinates near FP32's subnormal range: no far test
    }
    auto bucket = [&](const double xj, const double yj, const double zj, const double rj, int32_t j, int m) {
        double dx = xj - xi, dy = yj - yi, dz = zj - zi;
        if (periodic) {
            dx = mic64(dx, L, halfL);
            dy = mic64(dy, L, halfL);
            dz = mic64(dz, L, halfL);
        }
        if (contact_rn(dx * dx + dy * dy + dz * dz, ri + rj)) f(j, m);  // dist <= r_i + r_j
    };
    // PACKED: the slot's index and FP32 record are loaded together (one round of loads per candidate)
    auto candidate = [&](int32_t s, int m) {
        const int32_t j = sorted_idx[s];
        if (PACKED) {
            const float4 q = P32[s];
            if (!(i < j)) return;
            float ax = fabsf(q.x - qi.x), ay = fabsf(q.y - qi.y), az = fabsf(q.z - qi.z);
            if (periodic) {
                ax = fminf(ax, fabsf(ax - Lf));
                ay = fminf(ay, fabsf(ay - Lf));
                az = fminf(az, fabsf(az - Lf));
            }
            const float sf = fmaf(q.w, 1.f + 0x1p-18f, qi.w);
            if (fmaf(ax, ax, fmaf(ay, ay, az * az)) > sf * sf) return;  // clearly apart
            const double2 a = P[2 * s], b = P[2 * s + 1];
            bucket(a.x, a.y, b.x, b.y, j, m);
        } else {
            if (!(i < j)) return;
            bucket(x[j], y[j], z[j], r[j], j, m);
        }
    };
    // Neighbour cell c = 9 (di + 1) + 3 (dj + 1) + (dk + 1): its bucket, or -1 outside an open box.
    auto cell_hash = [&](int c) -> int32_t {
        int32_t nx = cx + c / 9 - 1, ny = cy + (c / 3) % 3 - 1, nz = cz + c % 3 - 1;
        if (periodic) {  // cx, cy, cz lie in [0, grid): one step wraps (= floor_mod)
            nx = wrap1(nx, p.grid);
            ny = wrap1(ny, p.grid);
            nz = wrap1(nz, p.grid);
        } else if (nx < 0 || ny < 0 || nz < 0 || nx >= p.grid || ny >= p.grid || nz >= p.grid) {
            return -1;
        }
        return hash_cell(nx, ny, nz, mask);
    };
    // Usual case: the 27 cells map to distinct buckets (kept in registers: static indices).
    {
        int32_t h[27];
#pragma unroll
        for (int c = 0; c < 27; ++c) h[c] = cell_hash(c);
        bool dup = false;
#pragma unroll
        for (int c = 1; c < 27; ++c)
#pragma unroll
            for (int m = 0; m < c; ++m) dup |= h[c] >= 0 && h[c] == h[m];
        if (!dup) {
            if (PACKED) {
                // the next cell's bucket range is loaded while this cell's candidates are tested, and
                // candidates are taken two at a time: the loop is bound by load latency, not arithmetic
                int32_t start = 0, end = 0;
                if (h[0] >= 0) {
                    start = bstart[h[0]];
                    end = bstart[h[0] + 1];
                }
#pragma unroll 1
                for (int c = 0; c < 27; ++c) {
                    int32_t ns = 0, ne = 0;
                    const int32_t hn = c + 1 < 27 ? cell_hash(c + 1) : -1;
                    if (hn >= 0) {
                        ns = bstart[hn];
                        ne = bstart[hn + 1];
                    }
                    if (end > n) end = n;  // :199-201
                    int32_t s = start;
#pragma unroll 1
                    for (; s + 1 < end; s += 2) {
                        candidate(s, 1);
                        candidate(s + 1, 1);
                    }
                    if (s < end) candidate(s, 1);
                    start = ns;
                    end = ne;
                }
            } else {
                for (int c = 0; c < 27; ++c) {
                    const int32_t hc = cell_hash(c);
                    if (hc < 0) continue;
                    const int32_t start = bstart[hc];
                    int32_t end = bstart[hc + 1];
                    if (end > n) end = n;  // :199-201
                    for (int32_t s = start; s < end; ++s) candidate(s, 1);
                }
            }
            return;
        }
    }
    // Tiny grids or colliding buckets: a bucket seen from several cells is
    // scanned once, its contacts counted with that multiplicity.
    int32_t hs[27];
    int nh = 0;
    int mult[27];
    for (int di = -1; di <= 1; ++di)
        for (int dj = -1; dj <= 1; ++dj)
            for (int dk = -1; dk <= 1; ++dk) {
                int32_t nx = cx + di, ny = cy + dj, nz = cz + dk;
                if (periodic) {
                    nx = floor_mod(nx, p.grid);
                    ny = floor_mod(ny, p.grid);
                    nz = floor_mod(nz, p.grid);
                } else if (nx < 0 || ny < 0 || nz < 0 || nx >= p.grid || ny >= p.grid || nz >= p.grid) {
                    continue;
                }
                const int32_t h = hash_cell(nx, ny, nz, mask);
                int q = 0;
                while (q < nh && hs[q] != h) ++q;
                if (q == nh) {
                    hs[nh] = h;
                    mult[nh] = 1;
                    ++nh;
                } else {
                    ++mult[q];
                }
            }
    for (int q = 0; q < nh; ++q) {
        const int32_t start = bstart[hs[q]];
        int32_t end = bstart[hs[q] + 1];
        if (end > n) end = n;  // :199-201
        for (int32_t s = start; s < end; ++s) candidate(s, mult[q]);
    }
}

// The droplets' positions and radii in bucket order: P[2 s] = (x, y), P[2 s + 1] = (z, r) of sorted_idx[s].
__global__ void bucket_positions_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                        const double *__restrict__ z, const double *__restrict__ r,
                                        const HashParams *__restrict__ hp, const int32_t *__restrict__ sorted_idx,
                                        double2 *__restrict__ P, float4 *__restrict__ P32) {
    if (!hp->valid) return;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int j = sorted_idx[s];
        const double xj = x[j], yj = y[j], zj = z[j], rj = r[j];
        P[2 * s] = make_double2(xj, yj);
        P[2 * s + 1] = make_double2(zj, rj);
        P32[s] = make_float4((float)xj, (float)yj, (float)zj, (float)rj);
    }
}

template <bool PACKED>
__global__ void count_pairs_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                   const double *__restrict__ z, const double *__restrict__ r,
                                   const double2 *__restrict__ P, const float4 *__restrict__ P32,
                                   const HashParams *__restrict__ hp, int periodic,
                                   double L, int32_t mask, const int32_t *__restrict__ bstart,
                                   const int32_t *__restrict__ sorted_idx, int32_t *__restrict__ pair_count,
                                   unsigned long long *__restrict__ raw) {
    const HashParams p = *hp;
    unsigned long long local_raw = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = p.valid ? sorted_idx[t] : t;  // bucket order (the buckets are filled when valid)
        int32_t c = 0;
        if (p.valid) {
            for_each_contact<PACKED>(i, t, x, y, z, r, P, P32, p, periodic, L, 0.5 * L, mask, n, bstart,
                                     sorted_idx, [&](int32_t, int m) {
                                         ++c;
                                         local_raw += (unsigned long long)m;
                                     });
        }
        pair_count[i] = c;
    }
    if (local_raw) atomicAdd(raw, local_raw);
}

// Count pass of the context entry point: one warp per occupied bucket.  The
// droplets of a bucket share their 27 neighbour buckets when they lie in one
// cell (the usual case), so the warp loads the 27 bucket ranges once, lays
// their candidates out as one list and tests 32 candidates at a time, each lane
// against every droplet of the bucket (staged in shared memory): the lanes stay
// converged and each candidate is read once per bucket, not once per droplet.
// A bucket holding droplets of several cells (hash aliasing) is taken one cell
// at a time.  The tests are for_each_contact's (the FP32 far test, then the same
// FP64 contact test); a cell with a neighbour bucket seen from two of its
// neighbour cells, and a bucket of more than 32 droplets, take for_each_contact
// per droplet.  Counts per droplet do not depend on the order.
constexpr int CB_WARPS = 4;
constexpr int CB_LIST = 256;  // candidate slots staged per warp (more: found by search)
#ifndef CB_MIN_CTAS
#define CB_MIN_CTAS 8  // resident CTAs per SM the count pass is compiled for (latency-bound: more warps)
#endif

__global__ void __launch_bounds__(32 * CB_WARPS, CB_MIN_CTAS)
    count_pairs_bucket_kernel(int n, int table, const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const double *__restrict__ r,
                              const double2 *__restrict__ P, const float4 *__restrict__ P32,
                              const HashParams *__restrict__ hp, int periodic, double L, int32_t mask,
                              const int32_t *__restrict__ bstart, const int32_t *__restrict__ sorted_idx,
                              const int32_t *__restrict__ cell_xyz, int32_t *__restrict__ pair_count,
                              unsigned long long *__restrict__ raw) {
    __shared__ float4 s_q[CB_WARPS][32];                       // FP32 record, radius widened (far test)
    __shared__ double2 s_a[CB_WARPS][32], s_b[CB_WARPS][32];  // FP64 (x, y), (z, r)
    __shared__ int s_i[CB_WARPS][32], s_cnt[CB_WARPS][32], s_st[CB_WARPS][32], s_pre[CB_WARPS][32];
    __shared__ int s_list[CB_WARPS][CB_LIST];  // the cell's candidate slots (when they fit)
    const HashParams p = *hp;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    if (!p.valid) {
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) pair_count[t] = 0;
        return;
    }
    const double halfL = 0.5 * L;
    const float Lf = (float)L;
    unsigned long long local_raw = 0;
    const int warps_total = gridDim.x * CB_WARPS;
    for (long long g = (long long)blockIdx.x * CB_WARPS + wp; g * 32 < table; g += warps_total) {
        const long long bb = g * 32 + lane;
        int t0 = 0, m = 0;
        if (bb < table) {
            t0 = bstart[bb];
            m = bstart[bb + 1] - t0;
        }
        unsigned occ = __ballot_sync(0xffffffffu, m > 0);
        while (occ) {
            const int src = __ffs(occ) - 1;
            occ &= occ - 1;
            const int bt0 = __shfl_sync(0xffffffffu, t0, src), bm = __shfl_sync(0xffffffffu, m, src);
            if (bm > 32) {  // a crowded bucket: per droplet
                for (int k = lane; k < bm; k += 32) {
                    const int t = bt0 + k;
                    const int ii = sorted_idx[t];
                    int32_t c = 0;
                    for_each_contact<true>(ii, t, x, y, z, r, P, P32, p, periodic, L, halfL, mask, n, bstart,
                                           sorted_idx, [&](int32_t, int mult) {
                                               ++c;
                                               local_raw += (unsigned long long)mult;
                                           });
                    pair_count[ii] = c;
                }
                continue;
            }
            // the bucket's droplets, one per lane, grouped by cell (a bucket can hold several cells)
            int i = -1;
            int32_t cx = 0, cy = 0, cz = 0;
            double2 a = make_double2(0.0, 0.0), b = a;
            if (lane < bm) {
                const int t = bt0 + lane;
                i = sorted_idx[t];
                a = P[2 * t];
                b = P[2 * t + 1];
                cx = cell_xyz[i];  // cell_coord of the droplet (assign_kernel)
                cy = cell_xyz[n + i];
                cz = cell_xyz[2 * (size_t)n + i];
            }
            // lanes of the same cell (cell coordinates are >= 0; idle lanes get distinct negative x)
            const unsigned same_cell = __match_any_sync(0xffffffffu, lane < bm ? cx : -1 - lane) &
                                       __match_any_sync(0xffffffffu, cy) & __match_any_sync(0xffffffffu, cz);
            unsigned todo = __ballot_sync(0xffffffffu, lane < bm);
            while (todo) {
                const int leader = __ffs(todo) - 1;
                const unsigned grp = __shfl_sync(0xffffffffu, same_cell, leader);
                todo &= ~grp;
                const bool mine = (grp >> lane) & 1u;
                const int32_t cx0 = __shfl_sync(0xffffffffu, cx, leader), cy0 = __shfl_sync(0xffffffffu, cy, leader),
                              cz0 = __shfl_sync(0xffffffffu, cz, leader);
                // neighbour cell c = lane: 9 (di + 1) + 3 (dj + 1) + (dk + 1), as in for_each_contact
                int32_t h = -1;
                if (lane < 27) {
                    int32_t nx = cx0 + lane / 9 - 1, ny = cy0 + (lane / 3) % 3 - 1, nz = cz0 + lane % 3 - 1;
                    if (periodic) {
                        h = hash_cell(wrap1(nx, p.grid), wrap1(ny, p.grid), wrap1(nz, p.grid), mask);
                    } else if (!(nx < 0 || ny < 0 || nz < 0 || nx >= p.grid || ny >= p.grid || nz >= p.grid)) {
                        h = hash_cell(nx, ny, nz, mask);
                    }
                }
                const unsigned peers = __match_any_sync(0xffffffffu, lane < 27 ? h : -2 - lane);
                if (__any_sync(0xffffffffu, lane < 27 && h >= 0 && __popc(peers) > 1)) {
                    // a neighbour bucket seen from two cells: per droplet, with multiplicities
                    if (mine) {
                        const int t = bt0 + lane;
                        int32_t c = 0;
                        for_each_contact<true>(i, t, x, y, z, r, P, P32, p, periodic, L, halfL, mask, n, bstart,
                                               sorted_idx, [&](int32_t, int mult) {
                                                   ++c;
                                                   local_raw += (unsigned long long)mult;
                                               });
                        pair_count[i] = c;
                    }
                    continue;
                }
                int st = 0, len = 0;
                if (h >= 0) {
                    st = bstart[h];
                    int e = bstart[h + 1];
                    if (e > n) e = n;  // :199-201
                    len = e > st ? e - st : 0;
                }
                int inc = len;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += v;
                }
                const int total = __shfl_sync(0xffffffffu, inc, 31);
                const int gm = __popc(grp);
                s_st[wp][lane] = st;
                s_pre[wp][lane] = inc - len;
                const bool listed = total <= CB_LIST;
                if (listed)
                    for (int e = 0; e < len; ++e) s_list[wp][inc - len + e] = st + e;
                if (mine) {  // the group's droplets at slots 0 .. gm - 1
                    const int slot = __popc(grp & ((1u << lane) - 1u));
                    const float marg = (float)(0x1p-17 * (fmax(fabs(a.x), fmax(fabs(a.y), fabs(b.x))) + fabs(L)));
                    float4 q = P32[bt0 + lane];
                    q.w = q.w * (1.f + 0x1p-18f) + marg;  // as for_each_contact's qi
                    if (!(marg >= 0x1p-100f)) q.w = INFINITY;
                    s_q[wp][slot] = q;
                    s_a[wp][slot] = a;
                    s_b[wp][slot] = b;
                    s_i[wp][slot] = i;
                    s_cnt[wp][slot] = 0;
                }
                __syncwarp();
                const int *wi = s_i[wp];
                const float4 *wq = s_q[wp];
                for (int t = lane; t - lane < total; t += 32) {  // every lane takes the same number of rounds
                    if (t >= total) continue;
                    int sl;
                    if (listed) {
                        sl = s_list[wp][t];
                    } else {  // the neighbour bucket holding list entry t: the last c with s_pre[c] <= t
                        int lo = 0, hi = 26;
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (s_pre[wp][mid] <= t)
                                lo = mid;
                            else
                                hi = mid - 1;
                        }
                        sl = s_st[wp][lo] + (t - s_pre[wp][lo]);
                    }
                    const int32_t j = sorted_idx[sl];
                    const float4 q = P32[sl];
                    const float qw = q.w * (1.f + 0x1p-18f);
#pragma unroll 4
                    for (int k = 0; k < gm; ++k) {
                        const float4 qi = wq[k];
                        float ax = fabsf(q.x - qi.x), ay = fabsf(q.y - qi.y), az = fabsf(q.z - qi.z);
                        if (periodic) {
                            ax = fminf(ax, fabsf(ax - Lf));
                            ay = fminf(ay, fabsf(ay - Lf));
                            az = fminf(az, fabsf(az - Lf));
                        }
                        const float sf = qw + qi.w;
                        // i < j, and not clearly apart: the exact test (rare)
                        if (!(wi[k] < j) || fmaf(ax, ax, fmaf(ay, ay, az * az)) > sf * sf) continue;
                        const double2 ca = P[2 * sl], cb = P[2 * sl + 1];
                        const double2 ka = s_a[wp][k], kb = s_b[wp][k];
                        double dx = ca.x - ka.x, dy = ca.y - ka.y, dz = cb.x - kb.x;
                        if (periodic) {
                            dx = mic64(dx, L, halfL);
                            dy = mic64(dy, L, halfL);
                            dz = mic64(dz, L, halfL);
                        }
                        if (contact_rn(dx * dx + dy * dy + dz * dz, kb.y + cb.y)) {  // dist <= r_i + r_j
                            atomicAdd(&s_cnt[wp][k], 1);
                            ++local_raw;
                        }
                    }
                }
                __syncwarp();
                if (lane < gm) pair_count[s_i[wp][lane]] = s_cnt[wp][lane];
                __syncwarp();  // shared memory is rewritten by the next group
            }
        }
    }
    if (local_raw) atomicAdd(raw, local_raw);
}

template <bool PACKED>
__global__ void write_pairs_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                   const double *__restrict__ z, const double *__restrict__ r,
                                   const double2 *__restrict__ P, const float4 *__restrict__ P32,
                                   const HashParams *__restrict__ hp, int periodic, double L, int32_t mask,
                                   const int32_t *__restrict__ bstart, const int32_t *__restrict__ sorted_idx,
                                   const int64_t *__restrict__ offset, int32_t *__restrict__ pairs, int64_t cap,
                                   int64_t *__restrict__ counts, uint32_t *err) {
    const HashParams p = *hp;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counts[0] = p.valid ? offset[n] : 0;
        if (p.valid && offset[n] > cap) raise_device_error(err, DEM_DEVERR_PAIR_OVERFLOW);
    }
    if (!p.valid) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = sorted_idx[t];  // bucket order, as in count_pairs_kernel
        const int64_t o0 = offset[i], o1 = offset[i + 1];
        // the row's slots that fit in the buffer: all of them, except in the one row that the
        // capacity cuts (o0 < cap < o1), and none in the rows after it
        const int64_t m = (o1 < cap ? o1 : cap) - o0;
        if (m <= 0) continue;
        // ascending j within the row of droplet i: each j found is inserted into the sorted run
        // pairs[o0 .. o0 + len); once the run holds m entries the largest drops out, so a cut row
        // keeps its m smallest j and the buffer holds the lexicographically first cap pairs
        int64_t len = 0;
        for_each_contact<PACKED>(i, t, x, y, z, r, P, P32, p, periodic, L, 0.5 * L, mask, n, bstart, sorted_idx,
                                 [&](int32_t j, int) {
            int64_t q;
            if (len < m) {
                pairs[2 * (o0 + len)] = i;
                q = len++;
            } else {
                if (j >= pairs[2 * (o0 + m - 1) + 1]) return;
                q = m - 1;
            }
            while (q > 0 && pairs[2 * (o0 + q - 1) + 1] > j) {
                pairs[2 * (o0 + q) + 1] = pairs[2 * (o0 + q - 1) + 1];
                --q;
            }
            pairs[2 * (o0 + q) + 1] = j;
        });
    }
}

// DirectCollisionFrequency.compute, pbm/collision_frequency/direct_collision_freq.py:17-41, on the
// detected pairs: matrix[b_i][b_j] += 1 and matrix[b_j][b_i] += 1 for every pair.
__global__ void pair_bin_kernel(const int32_t *__restrict__ pairs, const int64_t *__restrict__ num_pairs,
                                int64_t cap, const int32_t *__restrict__ bins, int nbins,
                                unsigned int *__restrict__ matrix) {
    const int64_t k = min(num_pairs[0], cap);
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < k; p += (int64_t)gridDim.x * blockDim.x) {
        const int bi = bins[pairs[2 * p]], bj = bins[pairs[2 * p + 1]];
        atomicAdd(&matrix[bi * nbins + bj], 1u);
        atomicAdd(&matrix[bj * nbins + bi], 1u);
    }
}

int launch_hash_detect(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                       double L, int periodic, int table_size, int32_t *pairs, int64_t cap, int64_t *counts,
                       cudaStream_t s, int even_cells) {
    int rc = dem_ensure_table(ctx, table_size);
    if (rc) return rc;
    unsigned long long *slot = reinterpret_cast<unsigned long long *>(ctx->dscratch) + 2;
    HashParams *hp = reinterpret_cast<HashParams *>(ctx->dscratch + 4);
    const int32_t mask = table_size - 1;
    const int grid = max(1, min(ceil_div(n, 256), 8 * ctx->sm_count));
    rc = dem_check_cuda(ctx, cudaMemsetAsync(slot, 0, sizeof(unsigned long long), s), "memset");
    if (!rc) rc = dem_check_cuda(ctx, cudaMemsetAsync(counts, 0, 2 * sizeof(int64_t), s), "memset");
    if (!rc) rc = dem_check_cuda(ctx, cudaMemsetAsync(ctx->bucket_count, 0, sizeof(int32_t) * table_size, s), "memset");
    if (rc) return rc;
    if (n == 0) return DEM_OK;
    dem_prof_begin(ctx, "hash_detect", s);
    max_kernel<<<grid, 256, 0, counted(s)>>>(n, r, slot);
    hash_params_kernel<<<1, 1, 0, counted(s)>>>(slot, L, even_cells, hp);
    assign_kernel<<<grid, 256, 0, counted(s)>>>(n, x, y, z, hp, periodic, mask, ctx->cell_hash, ctx->bucket_count,
                                                ctx->cell_xyz);
    rc = dem_check_launch(ctx, "hash assign");
    if (rc) return rc;
    rc = exclusive_scan<int32_t, int32_t>(ctx, ctx->bucket_count, ctx->bucket_start, table_size, s);
    if (rc) return rc;
    rc = dem_check_cuda(ctx, cudaMemcpyAsync(ctx->bucket_cursor, ctx->bucket_start, sizeof(int32_t) * table_size,
                                             cudaMemcpyDeviceToDevice, s),
                        "cursor copy");
    if (rc) return rc;
    scatter_kernel<<<grid, 256, 0, counted(s)>>>(n, ctx->cell_hash, hp, ctx->bucket_cursor, ctx->sorted_idx);
    bucket_positions_kernel<<<grid, 256, 0, counted(s)>>>(n, x, y, z, r, hp, ctx->sorted_idx, ctx->hash_pos,
                                                          ctx->hash_pos32);
    const int dgrid = ceil_div(n, 128);
    const int cgrid = max(1, min(ceil_div(table_size, 32 * CB_WARPS), 32 * ctx->sm_count));
    count_pairs_bucket_kernel<<<cgrid, 32 * CB_WARPS, 0, counted(s)>>>(
        n, table_size, x, y, z, r, ctx->hash_pos, ctx->hash_pos32, hp, periodic, L, mask, ctx->bucket_start,
        ctx->sorted_idx, ctx->cell_xyz, ctx->pair_count, reinterpret_cast<unsigned long long *>(counts + 1));
    rc = dem_check_launch(ctx, "hash count");
    if (rc) return rc;
    rc = exclusive_scan<int32_t, int64_t>(ctx, ctx->pair_count, ctx->pair_offset, n, s);
    if (rc) return rc;
    write_pairs_kernel<true><<<dgrid, 128, 0, counted(s)>>>(n, x, y, z, r, ctx->hash_pos, ctx->hash_pos32, hp,
                                                            periodic, L, mask,
                                                            ctx->bucket_start, ctx->sorted_idx, ctx->pair_offset,
                                                            pairs, cap, counts, ctx->d_err);
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "hash write");
}

}  // namespace dem

// ===========================================================================
// Allocation-free variant of the spatial-hash detector.
//
// Some callers cannot call cudaMalloc at the time they detect collisions: a
// host application that hands the library a fixed device-memory budget up
// front and forbids later allocations, a control loop that must not take the
// device-wide synchronisation and latency jitter of cudaMalloc/cudaFree
// between steps, or code that runs while another component owns the CUDA
// allocator.  For them dem_hash_detect_noalloc needs no context and allocates
// nothing: its workspace (bucket table, per-droplet hashes, bucket members,
// per-droplet pair counts and offsets, scan totals) is the file-scope device
// array below, sized for at most NOALLOC_MAX_N droplets and a hash table of at
// most NOALLOC_MAX_TABLE buckets.  Every GPU that loads the library keeps this
// array (about 2.9 MB) until the process exits.
// ===========================================================================
#include <mutex>

namespace dem {

constexpr int NOALLOC_MAX_N = 65536;
constexpr int NOALLOC_MAX_TABLE = 131072;  // next power of two >= 2 * NOALLOC_MAX_N
constexpr int NOALLOC_MAX_DEVICES = 64;

constexpr size_t na_align(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t NA_CELL = 0;                                                      // int32[MAX_N]
constexpr size_t NA_SORTED = NA_CELL + na_align(sizeof(int32_t) * NOALLOC_MAX_N);    // int32[MAX_N]
constexpr size_t NA_PCOUNT = NA_SORTED + na_align(sizeof(int32_t) * NOALLOC_MAX_N);  // int32[MAX_N + 1]
constexpr size_t NA_POFF = NA_PCOUNT + na_align(sizeof(int32_t) * (NOALLOC_MAX_N + 1));       // int64[MAX_N + 1]
constexpr size_t NA_BCOUNT = NA_POFF + na_align(sizeof(int64_t) * (NOALLOC_MAX_N + 1));       // int32[MAX_TABLE]
constexpr size_t NA_BSTART = NA_BCOUNT + na_align(sizeof(int32_t) * NOALLOC_MAX_TABLE);       // int32[MAX_TABLE + 1]
constexpr size_t NA_BCURSOR = NA_BSTART + na_align(sizeof(int32_t) * (NOALLOC_MAX_TABLE + 1));  // int32[MAX_TABLE]
constexpr size_t NA_SUMS = NA_BCURSOR + na_align(sizeof(int32_t) * NOALLOC_MAX_TABLE);  // int64[SCAN_MAX_BLOCKS + 1]
constexpr size_t NA_MISC = NA_SUMS + na_align(sizeof(int64_t) * (SCAN_MAX_BLOCKS + 1));  // max slot, params, err
constexpr size_t NA_BYTES = NA_MISC + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

struct NoallocDevice {
    unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int sm_count = 0;
};
static NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mutex;

// Once per device, with that device current: the device address of the array.
// (In host code g_noalloc_scratch names a host-side stand-in, not device memory.)
static int noalloc_setup(NoallocDevice &out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DEM_E_CUDA;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return DEM_E_INVALID;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoallocDevice &d = g_noalloc_dev[dev];
    if (!d.scratch) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DEM_E_CUDA;
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return DEM_E_CUDA;
        d.sm_count = sms > 0 ? sms : 1;
        d.scratch = static_cast<unsigned char *>(p);
    }
    out = d;
    return DEM_OK;
}

}  // namespace dem

extern "C" int dem_hash_detect_noalloc(int n, const double *x, const double *y, const double *z, const double *r,
                                       double L, int periodic, int table_size, int32_t *pairs,
                                       int64_t pair_capacity, int64_t *counts, void *stream) {
    using namespace dem;
    if (n < 0 || n > NOALLOC_MAX_N) return DEM_E_CAPACITY;
    if (table_size < 1 || table_size > NOALLOC_MAX_TABLE || (table_size & (table_size - 1))) return DEM_E_CAPACITY;
    if (!counts || pair_capacity < 0 || (pair_capacity > 0 && !pairs)) return DEM_E_INVALID;
    if (n > 0 && (!x || !y || !z || !r)) return DEM_E_INVALID;
    NoallocDevice d;
    int rc = noalloc_setup(d);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *base = d.scratch;
    int32_t *cell_hash = reinterpret_cast<int32_t *>(base + NA_CELL);
    int32_t *sorted_idx = reinterpret_cast<int32_t *>(base + NA_SORTED);
    int32_t *pair_count = reinterpret_cast<int32_t *>(base + NA_PCOUNT);
    int64_t *pair_offset = reinterpret_cast<int64_t *>(base + NA_POFF);
    int32_t *bucket_count = reinterpret_cast<int32_t *>(base + NA_BCOUNT);
    int32_t *bucket_start = reinterpret_cast<int32_t *>(base + NA_BSTART);
    int32_t *bucket_cursor = reinterpret_cast<int32_t *>(base + NA_BCURSOR);
    void *sums = base + NA_SUMS;
    unsigned long long *slot = reinterpret_cast<unsigned long long *>(base + NA_MISC);
    HashParams *hp = reinterpret_cast<HashParams *>(base + NA_MISC + 16);
    uint32_t *err = reinterpret_cast<uint32_t *>(base + NA_MISC + 64);
    const int32_t mask = table_size - 1;
    const int grid = max(1, min(ceil_div(n, 256), 8 * d.sm_count));
    // the array keeps the previous call's contents: reset what must start at zero
    if (cudaMemsetAsync(base + NA_MISC, 0, 256, s) != cudaSuccess) return DEM_E_CUDA;
    if (cudaMemsetAsync(counts, 0, 2 * sizeof(int64_t), s) != cudaSuccess) return DEM_E_CUDA;
    if (cudaMemsetAsync(bucket_count, 0, sizeof(int32_t) * table_size, s) != cudaSuccess) return DEM_E_CUDA;
    if (n == 0) return DEM_OK;
    max_kernel<<<grid, 256, 0, counted(s)>>>(n, r, slot);
    hash_params_kernel<<<1, 1, 0, counted(s)>>>(slot, L, 0, hp);
    assign_kernel<<<grid, 256, 0, counted(s)>>>(n, x, y, z, hp, periodic, mask, cell_hash, bucket_count, nullptr);
    if (cudaGetLastError() != cudaSuccess) return DEM_E_CUDA;
    if (exclusive_scan_into<int32_t, int32_t>(bucket_count, bucket_start, table_size, static_cast<int32_t *>(sums),
                                              s) != cudaSuccess)
        return DEM_E_CUDA;
    if (cudaMemcpyAsync(bucket_cursor, bucket_start, sizeof(int32_t) * table_size, cudaMemcpyDeviceToDevice, s) !=
        cudaSuccess)
        return DEM_E_CUDA;
    scatter_kernel<<<grid, 256, 0, counted(s)>>>(n, cell_hash, hp, bucket_cursor, sorted_idx);
    const int dgrid = ceil_div(n, 128);
    count_pairs_kernel<false><<<dgrid, 128, 0, counted(s)>>>(n, x, y, z, r, nullptr, nullptr, hp, periodic, L, mask,
                                                             bucket_start, sorted_idx, pair_count,
                                                             reinterpret_cast<unsigned long long *>(counts + 1));
    if (cudaGetLastError() != cudaSuccess) return DEM_E_CUDA;
    if (exclusive_scan_into<int32_t, int64_t>(pair_count, pair_offset, n, static_cast<int64_t *>(sums), s) !=
        cudaSuccess)
        return DEM_E_CUDA;
    write_pairs_kernel<false><<<dgrid, 128, 0, counted(s)>>>(n, x, y, z, r, nullptr, nullptr, hp, periodic, L, mask,
                                                             bucket_start, sorted_idx, pair_offset, pairs,
                                                             pair_capacity, counts, err);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_E_CUDA;
}

extern "C" int dem_pair_bin_matrix(dem_ctx *ctx, const int32_t *pairs, const int64_t *num_pairs, int64_t pair_capacity,
                                   const int32_t *bins, int nbins, uint32_t *matrix, void *stream) {
    if (!ctx || nbins < 1 || !matrix || !num_pairs || pair_capacity < 0) return DEM_E_INVALID;
    if (pair_capacity > 0 && (!pairs || !bins)) return DEM_E_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = dem_check_cuda(ctx, cudaMemsetAsync(matrix, 0, sizeof(uint32_t) * nbins * nbins, s), "memset");
    if (rc || pair_capacity == 0) return rc;
    const int grid = (int)std::min<int64_t>((pair_capacity + 255) / 256, 8LL * ctx->sm_count);
    dem::pair_bin_kernel<<<grid, 256, 0, counted(s)>>>(pairs, num_pairs, pair_capacity, bins, nbins, matrix);
    return dem_check_launch(ctx, "pair bin matrix");
}
