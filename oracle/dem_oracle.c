/*
 * dem_oracle.c -- CPU restatement of the reference's DEM droplet hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA product is
 * compared against, and the timed CPU baseline ("port") in bench.py.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * legs load it.  The product never calls into it.
 *
 * Every function restates one reference function, in the reference's own
 * expression order, in IEEE binary64 with no contraction (-ffp-contract=off):
 *
 *   direct forces       dem/force_calculator/direct_droplet_force_calculator.py:183-253
 *   direct convection   dem/force_calculator/direct_droplet_force_calculator.py:354-411
 *   euler update        dem/solver/euler_droplet_solver.py:121-131 (numpy semantics)
 *   spatial hash        dem/collision_detector/spatial_hash_collision_detector.py:74-316
 *   merge               dem/solution/droplet_solution.py:208-287 (numpy semantics)
 *   flat octree         dem/octree/flat_tree.py:180-1612, dem/octree/octree_node.py:72-114
 *   periodic-image      dem/force_calculator/direct_droplet_force_calculator.py:128-182, :413-464
 *   Oseen correction    dem/octree/flat_tree.py:1070-1131, :1171-1213, :1271-1276
 *
 * Integer powers inside the reference's Taichi kernels (x**2, x**3, x**7) are
 * evaluated by exponentiation by squaring, the way Taichi lowers them:
 *   x**3 = x*(x*x),  x**7 = (x*(x*x))*((x*x)*(x*x)).
 * Python/numpy-scope powers (the merge) call libm pow(), as numpy does.
 * Parity with these restatements is pinned by tests/golden (the reference's
 * own classes run through a Taichi stand-in); the last bits of a real Taichi
 * LLVM run (fast-math contraction) are not pinned.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EXPORT __attribute__((visibility("default")))

static inline double ipow2(double x) { return x * x; }
static inline double ipow3(double x) { return x * (x * x); }
static inline double ipow7(double x) {
    double x2 = x * x;
    return (x * x2) * (x2 * x2);
}
static inline double ti_sign(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

/* Minimum image, direct_droplet_force_calculator.py:234-240 */
static inline double mic(double d, double L) {
    if (fabs(d) > L * 0.5) d -= ti_sign(d) * L;
    return d;
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

EXPORT int dem_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Direct O(N^2) dipole force: rows [i0, i1) of the full N x N sum.          */
/* direct_droplet_force_calculator.py:183-200 (_calculate_one_force) and     */
/* :202-253 (_calculate_forces).  j ascending, i != j, contact cut r > ri+rj */
/* ------------------------------------------------------------------------ */
EXPORT void dem_oracle_direct_forces(int n, const double *x, const double *y, const double *z,
                                     const double *r, double m_const, double L, int periodic,
                                     double *fx, double *fy, double *fz, int i0, int i1,
                                     int nthreads) {
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = i0; i < i1; ++i) {
        double Fx = 0.0, Fy = 0.0, Fz = 0.0;
        const double xi = x[i], yi = y[i], zi = z[i], ri = r[i];
        for (int j = 0; j < n; ++j) {
            if (i == j) continue;
            double dx = x[j] - xi, dy = y[j] - yi, dz = z[j] - zi;
            if (periodic) {
                dx = mic(dx, L);
                dy = mic(dy, L);
                dz = mic(dz, L);
            }
            const double r_mag = sqrt(ipow2(dx) + ipow2(dy) + ipow2(dz));
            const double r_sum = ri + r[j];
            if (r_mag > r_sum) {
                const double M = m_const * ipow3(ri) * ipow3(r[j]) / ipow7(r_mag);
                const double dx2 = ipow2(dx), dy2 = ipow2(dy), dz2 = ipow2(dz);
                const double fxy = M * (4 * dz2 - dx2 - dy2);
                Fx += fxy * dx;
                Fy += fxy * dy;
                Fz += M * (2 * dz2 - 3 * dx2 - 3 * dy2) * dz;
            }
        }
        fx[i] = Fx;
        fy[i] = Fy;
        fz[i] = Fz;
    }
}

/* ------------------------------------------------------------------------ */
/* Periodic-image Oseen correction on a regular n^3 grid (COMSOL lattice).   */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n;                    /* grid points per axis */
    const double *u, *v, *w;  /* n^3 values each, C order [ix][iy][iz] */
    double gmin, ginv;        /* first node, 1 / spacing */
    double Fz_inv, cL, eta_r; /* 1/Fz_comsol, L_comsol/L_sim, eta_comsol/eta_sim */
    double g_self;            /* self-image coefficient */
} ocorr;

/* _precompute_grid_idx, direct_droplet_force_calculator.py:146-163 (one axis) */
static inline void grid_idx(double x, double gmin, double inv_dx, int n, int *i, double *t) {
    double f = (x - gmin) * inv_dx;
    const double n_max = (double)(n - 1);
    f = f <= n_max ? f : n_max; /* ti.min(fx, n_max) */
    f = 0.0 >= f ? 0.0 : f;     /* ti.max(0.0, .)   */
    int k = (int)floor(f);
    if (k > n - 2) k = n - 2;
    *i = k;
    *t = f - (double)k;
}

/* _interp_precomp, :165-182: the eight corner terms summed in source order */
static inline double interp(const double *g, int n, int ix, int iy, int iz, double tx, double ty, double tz) {
#define G(a, b, c) g[((size_t)(ix + (a)) * n + (iy + (b))) * n + (iz + (c))]
    return G(0, 0, 0) * (1 - tx) * (1 - ty) * (1 - tz) + G(0, 0, 1) * (1 - tx) * (1 - ty) * tz +
           G(0, 1, 0) * (1 - tx) * ty * (1 - tz) + G(0, 1, 1) * (1 - tx) * ty * tz +
           G(1, 0, 0) * tx * (1 - ty) * (1 - tz) + G(1, 0, 1) * tx * (1 - ty) * tz +
           G(1, 1, 0) * tx * ty * (1 - tz) + G(1, 1, 1) * tx * ty * tz;
#undef G
}

/* The pair term, :413-457 (and flat_tree.py:1070-1131 / 1171-1213): the
 * full tensor from three permuted lookups, G_z(x,y,z), G_x(z,y,x),
 * G_y(x,z,y), contracted with F_j / Fz_comsol.  Adds to v in source order. */
static inline void corr_pair(const ocorr *c, double x, double y, double z, double fx, double fy, double fz,
                             double *v) {
    const double cL = c->cL;
    const double xc = x * cL, yc = y * cL, zc = z * cL;
    int ax, ay, az;
    double tx, ty, tz;
    grid_idx(xc, c->gmin, c->ginv, c->n, &ax, &tx);
    grid_idx(yc, c->gmin, c->ginv, c->n, &ay, &ty);
    grid_idx(zc, c->gmin, c->ginv, c->n, &az, &tz);
    const int n = c->n;
    const double gz_x = interp(c->u, n, ax, ay, az, tx, ty, tz);
    const double gz_y = interp(c->v, n, ax, ay, az, tx, ty, tz);
    const double gz_z = interp(c->w, n, ax, ay, az, tx, ty, tz);
    const double gx_x = interp(c->w, n, az, ay, ax, tz, ty, tx);
    const double gx_y = interp(c->v, n, az, ay, ax, tz, ty, tx);
    const double gx_z = interp(c->u, n, az, ay, ax, tz, ty, tx);
    const double gy_x = interp(c->u, n, ax, az, ay, tx, tz, ty);
    const double gy_y = interp(c->w, n, ax, az, ay, tx, tz, ty);
    const double gy_z = interp(c->v, n, ax, az, ay, tx, tz, ty);
    const double common = c->Fz_inv * c->eta_r * cL;
    const double sx = fx * common, sy = fy * common, sz = fz * common;
    v[0] += gx_x * sx + gy_x * sy + gz_x * sz;
    v[1] += gx_y * sx + gy_y * sy + gz_y * sz;
    v[2] += gx_z * sx + gy_z * sy + gz_z * sz;
}

/* ------------------------------------------------------------------------ */
/* Direct O(N^2) Oseen convection, direct_droplet_force_calculator.py:354-411 */
/* d = x_i - x_j, no contact cut, COMSOL correction off.                     */
/* ------------------------------------------------------------------------ */
EXPORT void dem_oracle_direct_convection(int n, const double *x, const double *y, const double *z,
                                         const double *fx, const double *fy, const double *fz,
                                         double eta_const, double L, int periodic, double *vx,
                                         double *vy, double *vz, int i0, int i1, int nthreads) {
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = i0; i < i1; ++i) {
        double Cx = 0.0, Cy = 0.0, Cz = 0.0;
        const double xi = x[i], yi = y[i], zi = z[i];
        for (int j = 0; j < n; ++j) {
            if (i == j) continue;
            double X = xi - x[j], Y = yi - y[j], Z = zi - z[j];
            if (periodic) {
                X = mic(X, L);
                Y = mic(Y, L);
                Z = mic(Z, L);
            }
            const double rr = sqrt(ipow2(X) + ipow2(Y) + ipow2(Z));
            const double Fx = fx[j], Fy = fy[j], Fz = fz[j];
            const double r3 = ipow3(rr);
            const double Vx =
                eta_const * ((1 / rr + (ipow2(X)) / r3) * Fx + (X * Y) / r3 * Fy + (X * Z) / r3 * Fz);
            const double Vy =
                eta_const * ((X * Y) / r3 * Fx + (1 / rr + (ipow2(Y)) / r3) * Fy + (Y * Z) / r3 * Fz);
            const double Vz =
                eta_const * ((X * Z) / r3 * Fx + (Y * Z) / r3 * Fy + (1 / rr + (ipow2(Z)) / r3) * Fz);
            Cx += Vx;
            Cy += Vy;
            Cz += Vz;
        }
        vx[i] = Cx;
        vy[i] = Cy;
        vz[i] = Cz;
    }
}

/* The same with the periodic-image correction enabled, :354-464: per pair the
 * Stokeslet term, then the correction term; after the loop the self term
 * g_self * F_i. */
EXPORT void dem_oracle_direct_convection_corr(int n, const double *x, const double *y, const double *z,
                                              const double *fx, const double *fy, const double *fz,
                                              double eta_const, double L, int periodic, int gn,
                                              const double *gu, const double *gv, const double *gw, double gmin,
                                              double ginv, double Fz_inv, double cL, double eta_r, double g_self,
                                              double *vx, double *vy, double *vz, int i0, int i1, int nthreads) {
    const ocorr c = {gn, gu, gv, gw, gmin, ginv, Fz_inv, cL, eta_r, g_self};
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = i0; i < i1; ++i) {
        double C[3] = {0.0, 0.0, 0.0};
        const double xi = x[i], yi = y[i], zi = z[i];
        for (int j = 0; j < n; ++j) {
            if (i == j) continue;
            double X = xi - x[j], Y = yi - y[j], Z = zi - z[j];
            if (periodic) {
                X = mic(X, L);
                Y = mic(Y, L);
                Z = mic(Z, L);
            }
            const double rr = sqrt(ipow2(X) + ipow2(Y) + ipow2(Z));
            const double Fx = fx[j], Fy = fy[j], Fz = fz[j];
            const double r3 = ipow3(rr);
            C[0] += eta_const * ((1 / rr + (ipow2(X)) / r3) * Fx + (X * Y) / r3 * Fy + (X * Z) / r3 * Fz);
            C[1] += eta_const * ((X * Y) / r3 * Fx + (1 / rr + (ipow2(Y)) / r3) * Fy + (Y * Z) / r3 * Fz);
            C[2] += eta_const * ((X * Z) / r3 * Fx + (Y * Z) / r3 * Fy + (1 / rr + (ipow2(Z)) / r3) * Fz);
            corr_pair(&c, X, Y, Z, Fx, Fy, Fz, C);
        }
        C[0] += g_self * fx[i];
        C[1] += g_self * fy[i];
        C[2] += g_self * fz[i];
        vx[i] = C[0];
        vy[i] = C[1];
        vz[i] = C[2];
    }
}

/* numpy's float remainder (npy_divmod): fmod, then shift negative results by L */
static inline double np_remainder(double a, double b) {
    double mod = fmod(a, b);
    if (mod != 0.0) {
        if ((b < 0) != (mod < 0)) mod += b;
    } else {
        mod = copysign(0.0, b);
    }
    return mod;
}

/* ------------------------------------------------------------------------ */
/* Euler update of the direct path, euler_droplet_solver.py:121-131          */
/*   v_mig = F / (stokes_factor * r);  x += (v_mig + v_conv) * dt;  x %= L   */
/* pos is (n,3) row-major like the reference's numpy array.                  */
/* ------------------------------------------------------------------------ */
EXPORT void dem_oracle_euler_direct(int n, double *pos, const double *r, const double *F,
                                    const double *V, double stokes_factor, double dt, double L,
                                    int periodic) {
    for (int i = 0; i < n; ++i) {
        const double denom = stokes_factor * r[i];
        for (int c = 0; c < 3; ++c) {
            const double mig = F[3 * i + c] / denom;
            double p = pos[3 * i + c] + (mig + V[3 * i + c]) * dt;
            if (periodic) p = np_remainder(p, L);
            pos[3 * i + c] = p;
        }
    }
}

/* Euler update of the tree path, euler_droplet_solver.py:119, :130-131 */
EXPORT void dem_oracle_euler_total(int n, double *pos, const double *Vt, double dt, double L,
                                   int periodic) {
    for (int i = 0; i < 3 * n; ++i) {
        double p = pos[i] + Vt[i] * dt;
        if (periodic) p = np_remainder(p, L);
        pos[i] = p;
    }
}

/* ------------------------------------------------------------------------ */
/* Spatial hash collision detection,                                        */
/* spatial_hash_collision_detector.py:74-316.  Positions (n,3) row-major.    */
/* Returns the number of unique pairs written to pairs_out (lexicographic,   */
/* i<j), or -needed if cap is too small.  *raw_count receives the number of  */
/* raw (possibly duplicated) hits the reference would append.               */
/* ------------------------------------------------------------------------ */
static inline int32_t hash_cell(int32_t ix, int32_t iy, int32_t iz, int32_t mask) {
    uint32_t h = ((uint32_t)ix * 73856093u) ^ ((uint32_t)iy * 19349663u) ^ ((uint32_t)iz * 83492791u);
    return (int32_t)(h & (uint32_t)mask);
}
static inline int32_t floor_mod(int32_t a, int32_t m) {
    int32_t q = a % m;
    return q < 0 ? q + m : q;
}
static inline void cell_of(const double *p, double cs, int32_t gd, int periodic, int32_t *c) {
    for (int a = 0; a < 3; ++a) {
        int32_t v = (int32_t)floor(p[a] / cs);
        if (periodic) {
            v = floor_mod(v, gd);
        } else {
            if (v < 0) v = 0;
            if (v >= gd) v = gd - 1;
        }
        c[a] = v;
    }
}

static int cmp_pair(const void *a, const void *b) {
    const int32_t *p = (const int32_t *)a, *q = (const int32_t *)b;
    if (p[0] != q[0]) return p[0] < q[0] ? -1 : 1;
    if (p[1] != q[1]) return p[1] < q[1] ? -1 : 1;
    return 0;
}

EXPORT int64_t dem_oracle_hash_detect(int n, const double *pos, const double *r, double L,
                                      int periodic, int table_size, int32_t *pairs_out, int64_t cap,
                                      int64_t *raw_count) {
    *raw_count = 0;
    if (n <= 0) return 0;
    double max_radius = r[0];
    for (int i = 1; i < n; ++i)
        if (r[i] > max_radius) max_radius = r[i];
    const double cs = 2.0 * max_radius;
    if (!(cs > 0)) return 0; /* :259-260 */
    int32_t gd = (int32_t)ceil(L / cs);
    if (gd < 1) gd = 1;
    const int32_t mask = table_size - 1;
    int32_t *count = calloc((size_t)table_size, sizeof(int32_t));
    int32_t *offset = calloc((size_t)table_size, sizeof(int32_t));
    int32_t *cursor = calloc((size_t)table_size, sizeof(int32_t));
    int32_t *pcell = malloc(sizeof(int32_t) * (size_t)n);
    int32_t *sorted = malloc(sizeof(int32_t) * (size_t)n);
    for (int i = 0; i < n; ++i) { /* _assign_cells :79-112 */
        int32_t c[3];
        cell_of(pos + 3 * i, cs, gd, periodic, c);
        pcell[i] = hash_cell(c[0], c[1], c[2], mask);
        count[pcell[i]]++;
    }
    int32_t running = 0; /* _prefix_sum :115-123 */
    for (int h = 0; h < table_size; ++h) {
        offset[h] = running;
        cursor[h] = running;
        running += count[h];
    }
    for (int i = 0; i < n; ++i) sorted[cursor[pcell[i]]++] = i; /* _scatter :126-132 */

    int64_t raw = 0, cap_raw = 64 + 4 * (int64_t)n;
    int32_t *buf = malloc(sizeof(int32_t) * 2 * (size_t)cap_raw);
    for (int i = 0; i < n; ++i) { /* _detect_collisions :135-229 */
        const double *pi = pos + 3 * i;
        const double ri = r[i];
        int32_t c[3];
        cell_of(pi, cs, gd, periodic, c);
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk) {
                    int32_t nx = c[0] + di, ny = c[1] + dj, nz = c[2] + dk;
                    if (periodic) {
                        nx = floor_mod(nx, gd);
                        ny = floor_mod(ny, gd);
                        nz = floor_mod(nz, gd);
                    } else if (nx < 0 || ny < 0 || nz < 0 || nx >= gd || ny >= gd || nz >= gd) {
                        continue;
                    }
                    const int32_t nh = hash_cell(nx, ny, nz, mask);
                    const int32_t start = offset[nh];
                    int32_t end = start + count[nh];
                    if (end > n) end = n;
                    for (int32_t s = start; s < end; ++s) {
                        const int32_t j = sorted[s];
                        if (!(i < j)) continue;
                        const double *pj = pos + 3 * j;
                        double dx = pj[0] - pi[0], dy = pj[1] - pi[1], dz = pj[2] - pi[2];
                        if (periodic) {
                            dx = mic(dx, L);
                            dy = mic(dy, L);
                            dz = mic(dz, L);
                        }
                        const double dist = sqrt(dx * dx + dy * dy + dz * dz);
                        const double r_sum = ri + r[j];
                        if (dist <= r_sum) {
                            if (raw == cap_raw) {
                                cap_raw *= 2;
                                buf = realloc(buf, sizeof(int32_t) * 2 * (size_t)cap_raw);
                            }
                            buf[2 * raw] = i;
                            buf[2 * raw + 1] = j;
                            raw++;
                        }
                    }
                }
    }
    qsort(buf, (size_t)raw, 2 * sizeof(int32_t), cmp_pair); /* np.unique(axis=0) :312 */
    int64_t u = 0;
    for (int64_t k = 0; k < raw; ++k) {
        if (u > 0 && buf[2 * k] == buf[2 * (u - 1)] && buf[2 * k + 1] == buf[2 * (u - 1) + 1]) continue;
        buf[2 * u] = buf[2 * k];
        buf[2 * u + 1] = buf[2 * k + 1];
        u++;
    }
    *raw_count = raw;
    int64_t ret = u;
    if (u > cap) {
        ret = -u;
    } else {
        memcpy(pairs_out, buf, sizeof(int32_t) * 2 * (size_t)u);
    }
    free(buf);
    free(count);
    free(offset);
    free(cursor);
    free(pcell);
    free(sorted);
    return ret;
}

/* ------------------------------------------------------------------------ */
/* Coalescence, droplet_solution.py:208-287.  Pairs are visited in the order */
/* given (the caller sorts them by (i, j)); greedy: skip a pair whose ends   */
/* already merged.  r_new = (r1^3 + r2^3)^(1/3), x_new = (x1 r1^3 + x2 r2^3) */
/* / (r1^3 + r2^3) without minimum image.  Survivors keep their order; the   */
/* merged droplets are appended in pair order.  Returns the new count.       */
/* ------------------------------------------------------------------------ */
EXPORT int dem_oracle_merge(int n, const double *pos, const double *r, const int32_t *pairs, int k,
                            double *out_pos, double *out_r, int32_t *merged_pairs_out) {
    char *used = calloc((size_t)(n > 0 ? n : 1), 1);
    double *np_ = malloc(sizeof(double) * 3 * (size_t)(k > 0 ? k : 1));
    double *nr = malloc(sizeof(double) * (size_t)(k > 0 ? k : 1));
    int m = 0;
    for (int p = 0; p < k; ++p) {
        const int a = pairs[2 * p], b = pairs[2 * p + 1];
        if (used[a] || used[b]) continue;
        const double c1 = pow(r[a], 3.0), c2 = pow(r[b], 3.0);
        nr[m] = pow(c1 + c2, 1.0 / 3.0);
        for (int c = 0; c < 3; ++c) np_[3 * m + c] = (pos[3 * a + c] * c1 + pos[3 * b + c] * c2) / (c1 + c2);
        if (merged_pairs_out) {
            merged_pairs_out[2 * m] = a;
            merged_pairs_out[2 * m + 1] = b;
        }
        used[a] = used[b] = 1;
        m++;
    }
    int w = 0;
    for (int i = 0; i < n; ++i) {
        if (used[i]) continue;
        out_r[w] = r[i];
        for (int c = 0; c < 3; ++c) out_pos[3 * w + c] = pos[3 * i + c];
        w++;
    }
    for (int q = 0; q < m; ++q, ++w) {
        out_r[w] = nr[q];
        for (int c = 0; c < 3; ++c) out_pos[3 * w + c] = np_[3 * q + c];
    }
    free(used);
    free(np_);
    free(nr);
    return w;
}

/* ======================================================================== */
/* Flat octree, dem/octree/flat_tree.py + octree_node.py                     */
/* ======================================================================== */
typedef struct {
    int cap, max_nodes, n, mpl, periodic;
    double L, theta_sq;
    /* node arrays (octree_node.py:29-70) */
    double *mnx, *mny, *mnz, *mxx, *mxy, *mxz;
    double *R3, *R3x, *R3y, *R3z, *maxr;
    double *fsx, *fsy, *fsz, *P; /* P: 9 per node, row a (x,y,z) col b */
    int32_t *first_child, *next, *leaf_start, *count;
    int32_t *parents, *parent_fc;
    int32_t (*child_cnt)[8];
    int32_t *leaf_idx, *part_node, *part_oct;
    int node_count, parent_count, leaf_slot_count;
    int level_off[64];
    int n_levels;
    double *px, *py, *pz, *pr, *pf; /* particles; pf (n,3) forces */
    int corr_on;                    /* load_periodic_correction, flat_tree.py:141-167 */
    ocorr corr;
} otree;

EXPORT void *dem_oracle_tree_create(int num_particles, int mpl, double theta, int max_nodes_override) {
    otree *t = calloc(1, sizeof(otree));
    int n = num_particles > 64 ? num_particles : 64; /* flat_tree.py:63 */
    int mn = 4 * n / (mpl > 1 ? mpl : 1);            /* flat_tree.py:66 */
    if (mn < 1024) mn = 1024;
    if (max_nodes_override > 0) mn = max_nodes_override;
    t->cap = n;
    t->max_nodes = mn;
    t->mpl = mpl;
    t->theta_sq = theta * theta;
#define A(f, T, k) t->f = calloc((size_t)(k), sizeof(T))
    A(mnx, double, mn); A(mny, double, mn); A(mnz, double, mn);
    A(mxx, double, mn); A(mxy, double, mn); A(mxz, double, mn);
    A(R3, double, mn); A(R3x, double, mn); A(R3y, double, mn); A(R3z, double, mn); A(maxr, double, mn);
    A(fsx, double, mn); A(fsy, double, mn); A(fsz, double, mn); A(P, double, 9 * (size_t)mn);
    A(first_child, int32_t, mn); A(next, int32_t, mn); A(leaf_start, int32_t, mn); A(count, int32_t, mn);
    A(parents, int32_t, mn); A(parent_fc, int32_t, mn);
    t->child_cnt = calloc((size_t)mn, sizeof(int32_t[8]));
    A(leaf_idx, int32_t, n); A(part_node, int32_t, n); A(part_oct, int32_t, n);
    A(px, double, n); A(py, double, n); A(pz, double, n); A(pr, double, n); A(pf, double, 3 * (size_t)n);
#undef A
    return t;
}

EXPORT void dem_oracle_tree_destroy(void *h) {
    otree *t = h;
    if (!t) return;
    void *ptrs[] = {t->mnx, t->mny, t->mnz, t->mxx, t->mxy, t->mxz, t->R3, t->R3x, t->R3y, t->R3z,
                    t->maxr, t->fsx, t->fsy, t->fsz, t->P, t->first_child, t->next, t->leaf_start,
                    t->count, t->parents, t->parent_fc, t->child_cnt, t->leaf_idx, t->part_node,
                    t->part_oct, t->px, t->py, t->pz, t->pr, t->pf};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
    free(t);
}

/* load_periodic_correction, flat_tree.py:141-167 (gn == 0 switches it off).
 * The grids are borrowed: they must outlive the tree's use of them. */
EXPORT void dem_oracle_tree_set_correction(void *h, int gn, const double *gu, const double *gv, const double *gw,
                                           double gmin, double ginv, double Fz_inv, double cL, double eta_r,
                                           double g_self) {
    otree *t = h;
    const ocorr c = {gn, gu, gv, gw, gmin, ginv, Fz_inv, cL, eta_r, g_self};
    t->corr = c;
    t->corr_on = gn > 0;
}

EXPORT void dem_oracle_tree_set_params(void *h, double theta, int mpl) {
    otree *t = h;
    t->theta_sq = theta * theta;
    t->mpl = mpl;
}

static void init_node(otree *t, int idx, double a, double b, double c, double d, double e, double f) {
    /* octree_node.py:117-154 */
    t->mnx[idx] = a; t->mny[idx] = b; t->mnz[idx] = c;
    t->mxx[idx] = d; t->mxy[idx] = e; t->mxz[idx] = f;
    t->first_child[idx] = -1; t->next[idx] = -1; t->leaf_start[idx] = -1; t->count[idx] = 0;
    t->R3[idx] = t->R3x[idx] = t->R3y[idx] = t->R3z[idx] = t->maxr[idx] = 0.0;
    t->fsx[idx] = t->fsy[idx] = t->fsz[idx] = 0.0;
    for (int k = 0; k < 9; ++k) t->P[9 * idx + k] = 0.0;
}

static inline int get_octant(const otree *t, int idx, double x, double y, double z) {
    /* octree_node.py:84-95 */
    const double cx = (t->mnx[idx] + t->mxx[idx]) * 0.5;
    const double cy = (t->mny[idx] + t->mxy[idx]) * 0.5;
    const double cz = (t->mnz[idx] + t->mxz[idx]) * 0.5;
    int o = 0;
    if (x >= cx) o |= 1;
    if (y >= cy) o |= 2;
    if (z >= cz) o |= 4;
    return o;
}

static inline double node_size(const otree *t, int idx) { /* octree_node.py:77-81 */
    double dx = t->mxx[idx] - t->mnx[idx], dy = t->mxy[idx] - t->mny[idx], dz = t->mxz[idx] - t->mnz[idx];
    double m = dx >= dy ? dx : dy;
    return m >= dz ? m : dz;
}

static inline void node_center(const otree *t, int idx, double *c) { /* octree_node.py:98-114 */
    if (t->R3[idx] > 0.0) {
        const double inv = 1.0 / t->R3[idx];
        c[0] = t->R3x[idx] * inv;
        c[1] = t->R3y[idx] * inv;
        c[2] = t->R3z[idx] * inv;
    } else {
        c[0] = (t->mnx[idx] + t->mxx[idx]) * 0.5;
        c[1] = (t->mny[idx] + t->mxy[idx]) * 0.5;
        c[2] = (t->mnz[idx] + t->mxz[idx]) * 0.5;
    }
}

/* FlatOctree.build, flat_tree.py:180-246 (+ phases :248-463, :469-554).
 * pos (n,3) row-major.  Returns 0, or -1 when n exceeds the capacity. */
EXPORT int dem_oracle_tree_build(void *h, int n, const double *pos, const double *r, double L,
                                 int periodic) {
    otree *t = h;
    if (n > t->cap) return -1;
    t->n = n;
    t->L = L;
    t->periodic = periodic ? 1 : 0;
    for (int i = 0; i < n; ++i) {
        t->px[i] = pos[3 * i];
        t->py[i] = pos[3 * i + 1];
        t->pz[i] = pos[3 * i + 2];
        t->pr[i] = r[i];
    }
    t->node_count = 1;
    t->parent_count = 0;
    t->leaf_slot_count = 0;
    int ls = 0, le = 1;
    /* _init_root_kernel :249-270 (fmom/max_radius are not reset there) */
    t->mnx[0] = t->mny[0] = t->mnz[0] = 0.0;
    t->mxx[0] = t->mxy[0] = t->mxz[0] = L;
    t->first_child[0] = -1; t->next[0] = -1; t->leaf_start[0] = -1; t->count[0] = n;
    t->R3[0] = t->R3x[0] = t->R3y[0] = t->R3z[0] = 0.0;
    t->fsx[0] = t->fsy[0] = t->fsz[0] = 0.0;
    for (int i = 0; i < n; ++i) t->part_node[i] = 0;
    t->n_levels = 0;
    for (int level = 0; level < 40; ++level) {
        int overflow = 0;
        const int pc_before = t->parent_count;
        /* _level_assign_octants :284-306 */
        for (int node = ls; node < le; ++node)
            for (int o = 0; o < 8; ++o) t->child_cnt[node][o] = 0;
        for (int i = 0; i < n; ++i) {
            const int node = t->part_node[i];
            if (node >= ls && node < le) {
                const int o = get_octant(t, node, t->px[i], t->py[i], t->pz[i]);
                t->part_oct[i] = o;
                t->child_cnt[node][o]++;
            }
        }
        /* _level_subdivide_and_alloc :309-354 */
        for (int node = ls; node < le; ++node) {
            if (t->first_child[node] < 0 && t->count[node] > t->mpl) {
                const int base = t->node_count;
                if (base + 8 > t->max_nodes) continue;
                t->node_count = base + 8;
                t->first_child[node] = base;
                const int p = t->parent_count;
                t->parents[p] = node;
                t->parent_fc[p] = base;
                t->parent_count = p + 1;
                const double cx = (t->mnx[node] + t->mxx[node]) * 0.5;
                const double cy = (t->mny[node] + t->mxy[node]) * 0.5;
                const double cz = (t->mnz[node] + t->mxz[node]) * 0.5;
                for (int o = 0; o < 8; ++o) {
                    const int child = base + o;
                    const double a = (o & 1) ? cx : t->mnx[node];
                    const double b = (o & 2) ? cy : t->mny[node];
                    const double c = (o & 4) ? cz : t->mnz[node];
                    const double d = (o & 1) ? t->mxx[node] : cx;
                    const double e = (o & 2) ? t->mxy[node] : cy;
                    const double f = (o & 4) ? t->mxz[node] : cz;
                    init_node(t, child, a, b, c, d, e, f);
                    t->count[child] = t->child_cnt[node][o];
                }
                overflow = 1;
            }
        }
        /* _level_scatter :357-366 */
        for (int i = 0; i < n; ++i) {
            const int node = t->part_node[i];
            if (node >= 0 && t->first_child[node] >= 0) t->part_node[i] = t->first_child[node] + t->part_oct[i];
        }
        ls = le;
        le = t->node_count;
        if (t->parent_count > pc_before) t->level_off[t->n_levels++] = pc_before;
        if (!overflow) break;
    }
    /* _finalize_leaves_alloc :371-385 */
    for (int node = 0; node < t->node_count; ++node) {
        if (t->first_child[node] < 0 && t->count[node] > 0) {
            const int cnt = t->count[node];
            t->leaf_start[node] = t->leaf_slot_count;
            t->leaf_slot_count += cnt;
            t->count[node] = 0;
        }
    }
    /* _finalize_leaves_scatter :388-397 (serial: ascending particle index) */
    for (int i = 0; i < n; ++i) {
        const int node = t->part_node[i];
        if (node >= 0 && t->first_child[node] < 0) {
            const int l0 = t->leaf_start[node];
            if (l0 >= 0) t->leaf_idx[l0 + t->count[node]++] = i;
        }
    }
    /* _build_next_pointers :400-463 */
    for (int lev = 0; lev < t->n_levels; ++lev) {
        const int a = t->level_off[lev], b = lev + 1 < t->n_levels ? t->level_off[lev + 1] : t->parent_count;
        for (int i = a; i < b; ++i) {
            const int parent = t->parents[i], base = t->parent_fc[i];
            const int pn = t->next[parent];
            for (int o = 0; o < 8; ++o) t->next[base + o] = (o == 7) ? pn : base + o + 1;
        }
    }
    for (int lev = 0; lev < t->n_levels; ++lev) {
        const int a = t->level_off[lev], b = lev + 1 < t->n_levels ? t->level_off[lev + 1] : t->parent_count;
        for (int i = a; i < b; ++i) {
            const int parent = t->parents[i], base = t->parent_fc[i];
            if (t->count[parent] == 0) {
                t->first_child[parent] = t->next[parent];
                continue;
            }
            int first = -1, last = -1;
            for (int j = 0; j < 8; ++j) {
                const int c = base + j;
                if (t->count[c] > 0) {
                    if (first < 0) {
                        first = last = c;
                    } else {
                        t->next[last] = c;
                        last = c;
                    }
                }
            }
            if (last >= 0) {
                t->next[last] = t->next[parent];
                t->first_child[parent] = first;
            }
        }
    }
    /* _propagate_r3: _init_leaf_r3 :470-511, _sweep_r3_level :514-542 */
    for (int idx = 0; idx < t->node_count; ++idx) {
        t->R3[idx] = t->R3x[idx] = t->R3y[idx] = t->R3z[idx] = t->maxr[idx] = 0.0;
        t->fsx[idx] = t->fsy[idx] = t->fsz[idx] = 0.0;
        if (t->first_child[idx] < 0 && t->count[idx] > 0 && t->leaf_start[idx] >= 0) {
            const int l0 = t->leaf_start[idx], cnt = t->count[idx];
            double s = 0, wx = 0, wy = 0, wz = 0, mr = 0;
            for (int k = 0; k < cnt; ++k) {
                const int p = t->leaf_idx[l0 + k];
                if (p >= 0) {
                    const double ri = t->pr[p];
                    const double r3 = ipow3(ri);
                    s += r3;
                    wx += t->px[p] * r3;
                    wy += t->py[p] * r3;
                    wz += t->pz[p] * r3;
                    if (ri > mr) mr = ri;
                }
            }
            t->R3[idx] = s;
            t->R3x[idx] = wx;
            t->R3y[idx] = wy;
            t->R3z[idx] = wz;
            t->maxr[idx] = mr;
        }
    }
    for (int lev = t->n_levels - 1; lev >= 0; --lev) {
        const int a = t->level_off[lev], b = lev + 1 < t->n_levels ? t->level_off[lev + 1] : t->parent_count;
        for (int i = a; i < b; ++i) {
            const int parent = t->parents[i], base = t->parent_fc[i];
            double s = 0, wx = 0, wy = 0, wz = 0, mr = 0;
            for (int j = 0; j < 8; ++j) {
                const int c = base + j;
                if (t->count[c] > 0) {
                    s += t->R3[c];
                    wx += t->R3x[c];
                    wy += t->R3y[c];
                    wz += t->R3z[c];
                    if (t->maxr[c] > mr) mr = t->maxr[c];
                }
            }
            t->R3[parent] = s;
            t->R3x[parent] = wx;
            t->R3y[parent] = wy;
            t->R3z[parent] = wz;
            t->maxr[parent] = mr;
        }
    }
    return 0;
}

/* _compute_forces_kernel, flat_tree.py:783-894.  Rows [i0, i1).  Also keeps
 * the forces for the Stokeslet propagation (particle_forces field).  f (n,3). */
EXPORT void dem_oracle_tree_forces(void *h, double m_const, double *f, int i0, int i1, int nthreads) {
    otree *t = h;
    set_threads(nthreads);
    const double th2 = t->theta_sq, L = t->L;
    const int per = t->periodic;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = i0; i < i1; ++i) {
        const double xi = t->px[i], yi = t->py[i], zi = t->pz[i];
        const double ri3 = ipow3(t->pr[i]);
        double Fx = 0, Fy = 0, Fz = 0;
        int node = 0;
        while (node >= 0) {
            const int cnt = t->count[node];
            if (cnt == 0 || t->R3[node] < 1e-30) {
                node = t->next[node];
                continue;
            }
            if (t->first_child[node] < 0) {
                const int l0 = t->leaf_start[node];
                for (int k = 0; k < cnt; ++k) {
                    const int j = t->leaf_idx[l0 + k];
                    if (j >= 0 && j != i) {
                        double dx = t->px[j] - xi, dy = t->py[j] - yi, dz = t->pz[j] - zi;
                        if (per) {
                            dx = mic(dx, L);
                            dy = mic(dy, L);
                            dz = mic(dz, L);
                        }
                        const double r_sq = dx * dx + dy * dy + dz * dz;
                        const double r_sum = t->pr[i] + t->pr[j];
                        if (r_sq >= r_sum * r_sum) {
                            const double rr = sqrt(r_sq);
                            const double r7 = r_sq * r_sq * r_sq * rr;
                            const double rj3 = ipow3(t->pr[j]);
                            const double factor = m_const * ri3 * rj3 / r7;
                            const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
                            const double ang = 4.0 * dz2 - dx2 - dy2;
                            Fx += factor * dx * ang;
                            Fy += factor * dy * ang;
                            Fz += factor * dz * (2.0 * dz2 - 3.0 * dx2 - 3.0 * dy2);
                        }
                    }
                }
                node = t->next[node];
                continue;
            }
            const double s = node_size(t, node);
            double c[3];
            node_center(t, node, c);
            double dx = c[0] - xi, dy = c[1] - yi, dz = c[2] - zi;
            if (per) {
                dx = mic(dx, L);
                dy = mic(dy, L);
                dz = mic(dz, L);
            }
            const double D_sq = dx * dx + dy * dy + dz * dz;
            if (s * s < th2 * D_sq && D_sq > 0.0) {
                const double rr = sqrt(D_sq);
                const double r7 = D_sq * D_sq * D_sq * rr;
                const double factor = m_const * ri3 * t->R3[node] / r7;
                const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
                const double ang = 4.0 * dz2 - dx2 - dy2;
                Fx += factor * dx * ang;
                Fy += factor * dy * ang;
                Fz += factor * dz * (2.0 * dz2 - 3.0 * dx2 - 3.0 * dy2);
                node = t->next[node];
            } else {
                node = t->first_child[node];
            }
        }
        f[3 * i] = Fx;
        f[3 * i + 1] = Fy;
        f[3 * i + 2] = Fz;
        t->pf[3 * i] = Fx;
        t->pf[3 * i + 1] = Fy;
        t->pf[3 * i + 2] = Fz;
    }
}

/* _propagate_forces_from_fields, flat_tree.py:696-777: leaf sums of F and of
 * the raw moments P_ab = sum x_a F_b, then a bottom-up sweep per level.  When
 * forces is non-NULL it replaces the kept particle forces (_propagate_forces,
 * :556-694, used by compute_stokeslet). */
EXPORT void dem_oracle_tree_propagate_forces(void *h, const double *forces) {
    otree *t = h;
    const double *F = forces ? forces : t->pf;
    for (int idx = 0; idx < t->node_count; ++idx) {
        t->fsx[idx] = t->fsy[idx] = t->fsz[idx] = 0.0;
        for (int k = 0; k < 9; ++k) t->P[9 * idx + k] = 0.0;
        if (t->first_child[idx] < 0 && t->count[idx] > 0 && t->leaf_start[idx] >= 0) {
            const int l0 = t->leaf_start[idx], cnt = t->count[idx];
            double s[3] = {0, 0, 0}, P[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int k = 0; k < cnt; ++k) {
                const int p = t->leaf_idx[l0 + k];
                if (p >= 0) {
                    const double f3[3] = {F[3 * p], F[3 * p + 1], F[3 * p + 2]};
                    const double x3[3] = {t->px[p], t->py[p], t->pz[p]};
                    s[0] += f3[0];
                    s[1] += f3[1];
                    s[2] += f3[2];
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) P[3 * a + b] += x3[a] * f3[b];
                }
            }
            t->fsx[idx] = s[0];
            t->fsy[idx] = s[1];
            t->fsz[idx] = s[2];
            for (int k = 0; k < 9; ++k) t->P[9 * idx + k] = P[k];
        }
    }
    for (int lev = t->n_levels - 1; lev >= 0; --lev) {
        const int a = t->level_off[lev], b = lev + 1 < t->n_levels ? t->level_off[lev + 1] : t->parent_count;
        for (int i = a; i < b; ++i) {
            const int parent = t->parents[i], base = t->parent_fc[i];
            double s[3] = {0, 0, 0}, P[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int j = 0; j < 8; ++j) {
                const int c = base + j;
                if (t->count[c] > 0) {
                    s[0] += t->fsx[c];
                    s[1] += t->fsy[c];
                    s[2] += t->fsz[c];
                    for (int k = 0; k < 9; ++k) P[k] += t->P[9 * c + k];
                }
            }
            t->fsx[parent] = s[0];
            t->fsy[parent] = s[1];
            t->fsz[parent] = s[2];
            for (int k = 0; k < 9; ++k) t->P[9 * parent + k] = P[k];
        }
    }
}

/* _compute_stokeslet_kernel (:1000-1280) when stokes_factor <= 0, else
 * _compute_total_velocity_kernel (:1326-1588).  forces (n,3): the array
 * passed as forces_np.  With a correction set (dem_oracle_tree_set_correction)
 * its pair terms follow every leaf pair and accepted node; the self term is
 * added by the Stokeslet walk only, as in the reference.  Rows [i0, i1). */
EXPORT void dem_oracle_tree_velocity(void *h, const double *forces, double eta_const,
                                     double stokes_factor, double *v, int i0, int i1, int nthreads) {
    otree *t = h;
    set_threads(nthreads);
    const double th2 = t->theta_sq, L = t->L;
    const int per = t->periodic;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = i0; i < i1; ++i) {
        const double xi = t->px[i], yi = t->py[i], zi = t->pz[i];
        double vx = 0, vy = 0, vz = 0;
        if (stokes_factor > 0) {
            const double inv_stokes_r = 1.0 / (stokes_factor * t->pr[i]);
            vx = t->pf[3 * i] * inv_stokes_r;
            vy = t->pf[3 * i + 1] * inv_stokes_r;
            vz = t->pf[3 * i + 2] * inv_stokes_r;
        }
        int node = 0;
        while (node >= 0) {
            const int cnt = t->count[node];
            const double fs2 = ipow2(t->fsx[node]) + ipow2(t->fsy[node]) + ipow2(t->fsz[node]);
            if (cnt == 0 || fs2 < 1e-60) {
                node = t->next[node];
                continue;
            }
            if (t->first_child[node] < 0) {
                const int l0 = t->leaf_start[node];
                for (int k = 0; k < cnt; ++k) {
                    const int j = t->leaf_idx[l0 + k];
                    if (j >= 0 && j != i) {
                        double dx = xi - t->px[j], dy = yi - t->py[j], dz = zi - t->pz[j];
                        if (per) {
                            dx = mic(dx, L);
                            dy = mic(dy, L);
                            dz = mic(dz, L);
                        }
                        const double r_sq = dx * dx + dy * dy + dz * dz;
                        const double r_sum = t->pr[i] + t->pr[j];
                        if (r_sq >= r_sum * r_sum) {
                            const double rr = sqrt(r_sq);
                            const double inv_r = 1.0 / rr;
                            const double inv_r2 = inv_r * inv_r;
                            const double Fx = forces[3 * j], Fy = forces[3 * j + 1], Fz = forces[3 * j + 2];
                            const double dot = dx * Fx + dy * Fy + dz * Fz;
                            const double coeff = eta_const * inv_r;
                            vx += coeff * (Fx + dx * inv_r2 * dot);
                            vy += coeff * (Fy + dy * inv_r2 * dot);
                            vz += coeff * (Fz + dz * inv_r2 * dot);
                            if (t->corr_on) { /* :1070-1131 */
                                double acc[3] = {vx, vy, vz};
                                corr_pair(&t->corr, dx, dy, dz, Fx, Fy, Fz, acc);
                                vx = acc[0];
                                vy = acc[1];
                                vz = acc[2];
                            }
                        }
                    }
                }
                node = t->next[node];
                continue;
            }
            const double s = node_size(t, node);
            double c[3];
            node_center(t, node, c);
            double dx = xi - c[0], dy = yi - c[1], dz = zi - c[2];
            if (per) {
                dx = mic(dx, L);
                dy = mic(dy, L);
                dz = mic(dz, L);
            }
            const double D_sq = dx * dx + dy * dy + dz * dz;
            if (s * s < th2 * D_sq && D_sq > 0.0) {
                const double rr = sqrt(D_sq);
                const double inv_r = 1.0 / rr;
                const double inv_r2 = inv_r * inv_r;
                const double Fx = t->fsx[node], Fy = t->fsy[node], Fz = t->fsz[node];
                const double dot = dx * Fx + dy * Fy + dz * Fz;
                const double coeff = eta_const * inv_r;
                vx += coeff * (Fx + dx * inv_r2 * dot);
                vy += coeff * (Fy + dy * inv_r2 * dot);
                vz += coeff * (Fz + dz * inv_r2 * dot);
                if (t->corr_on) { /* monopole term of the correction, :1171-1213 */
                    double acc[3] = {vx, vy, vz};
                    corr_pair(&t->corr, dx, dy, dz, Fx, Fy, Fz, acc);
                    vx = acc[0];
                    vy = acc[1];
                    vz = acc[2];
                }
                /* dipole correction :1215-1265 */
                const double r3s = t->R3[node];
                double cmx, cmy, cmz;
                if (r3s > 0.0) {
                    const double inv = 1.0 / r3s;
                    cmx = t->R3x[node] * inv;
                    cmy = t->R3y[node] * inv;
                    cmz = t->R3z[node] * inv;
                } else {
                    cmx = (t->mnx[node] + t->mxx[node]) * 0.5;
                    cmy = (t->mny[node] + t->mxy[node]) * 0.5;
                    cmz = (t->mnz[node] + t->mxz[node]) * 0.5;
                }
                const double *P = t->P + 9 * node;
                const double Dxx = P[0] - cmx * Fx, Dxy = P[1] - cmx * Fy, Dxz = P[2] - cmx * Fz;
                const double Dyx = P[3] - cmy * Fx, Dyy = P[4] - cmy * Fy, Dyz = P[5] - cmy * Fz;
                const double Dzx = P[6] - cmz * Fx, Dzy = P[7] - cmz * Fy, Dzz = P[8] - cmz * Fz;
                const double rx = dx, ry = dy, rz = dz;
                const double ux = Dxx * rx + Dyx * ry + Dzx * rz;
                const double uy = Dxy * rx + Dyy * ry + Dzy * rz;
                const double uz = Dxz * rx + Dyz * ry + Dzz * rz;
                const double wx = Dxx * rx + Dxy * ry + Dxz * rz;
                const double wy = Dyx * rx + Dyy * ry + Dyz * rz;
                const double wz = Dzx * rx + Dzy * ry + Dzz * rz;
                const double s_tr = Dxx + Dyy + Dzz;
                const double q = rx * wx + ry * wy + rz * wz;
                const double inv_r3 = inv_r * inv_r2;
                const double inv_r5 = inv_r3 * inv_r2;
                vx += eta_const * (inv_r3 * (ux - wx - s_tr * rx) + 3.0 * rx * q * inv_r5);
                vy += eta_const * (inv_r3 * (uy - wy - s_tr * ry) + 3.0 * ry * q * inv_r5);
                vz += eta_const * (inv_r3 * (uz - wz - s_tr * rz) + 3.0 * rz * q * inv_r5);
                node = t->next[node];
            } else {
                node = t->first_child[node];
            }
        }
        if (t->corr_on && !(stokes_factor > 0)) { /* self term, Stokeslet walk only (:1271-1276) */
            vx += t->corr.g_self * forces[3 * i];
            vy += t->corr.g_self * forces[3 * i + 1];
            vz += t->corr.g_self * forces[3 * i + 2];
        }
        v[3 * i] = vx;
        v[3 * i + 1] = vy;
        v[3 * i + 2] = vz;
    }
}

/* Structural introspection used by tests (node_count, parent_count, ...). */
EXPORT void dem_oracle_tree_stats(void *h, int64_t *out) {
    otree *t = h;
    out[0] = t->node_count;
    out[1] = t->parent_count;
    out[2] = t->leaf_slot_count;
    out[3] = t->max_nodes;
    out[4] = t->n_levels;
    out[5] = t->n;
}

EXPORT void dem_oracle_tree_nodes(void *h, int32_t *count, int32_t *first_child, int32_t *next,
                                  int32_t *leaf_start, double *r3, double *fs) {
    otree *t = h;
    for (int k = 0; k < t->node_count; ++k) {
        if (count) count[k] = t->count[k];
        if (first_child) first_child[k] = t->first_child[k];
        if (next) next[k] = t->next[k];
        if (leaf_start) leaf_start[k] = t->leaf_start[k];
        if (r3) {
            r3[4 * k] = t->R3[k];
            r3[4 * k + 1] = t->R3x[k];
            r3[4 * k + 2] = t->R3y[k];
            r3[4 * k + 3] = t->R3z[k];
        }
        if (fs) {
            fs[12 * k] = t->fsx[k];
            fs[12 * k + 1] = t->fsy[k];
            fs[12 * k + 2] = t->fsz[k];
            for (int q = 0; q < 9; ++q) fs[12 * k + 3 + q] = t->P[9 * k + q];
        }
    }
}

EXPORT void dem_oracle_tree_leaf_indices(void *h, int32_t *out) {
    otree *t = h;
    memcpy(out, t->leaf_idx, sizeof(int32_t) * (size_t)t->n);
}
