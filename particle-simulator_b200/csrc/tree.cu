// tree.cu -- flat Barnes-Hut octree (reference drop-in), FP64.
//
// Restates FlatOctree (dem/octree/flat_tree.py:36-1630, dem/octree/octree_node.py)
// on the device with the same tree, node numbering and arithmetic:
//   build            :180-246  level by level; the serial subdivision loop
//                              (:309-354) becomes a scan over the level's nodes
//                              (the first k candidates in node order get
//                              children, k limited by the node pool exactly as
//                              the serial `base + 8 > max_nodes` test does)
//   leaf slots       :371-397  leaves in node order, particles ascending inside
//   next pointers    :400-463  per level, top-down
//   R^3 aggregates   :469-554  leaves in particle order, parents in octant order
//   force walk       :783-894  stackless walk, MAC s^2 < theta^2 D^2
//   force moments    :696-777  sum F and P_ab = sum x_a F_b
//   velocity walks   :1000-1280 (Stokeslet) and :1326-1588 (total velocity)
// Every walk visits nodes in the reference's order and accumulates in the
// reference's order; the file is compiled with -fmad=false, so forces and
// velocities are bit-identical to the reference expressions in IEEE binary64.
#include <vector>

#include "common.cuh"
#include "corr.cuh"
#include "scan.cuh"

struct dem_tree {
    dem_ctx *ctx = nullptr;  // must outlive the tree while kernels run; destroy does not touch it
    int device = 0;
    int cap = 0, max_nodes = 0;
    int n = 0, node_count = 0, parent_count = 0, leaf_slot_count = 0, pool_exhausted = 0;
    double L = 0;
    int periodic = 0;
    std::vector<int> level_off;
    // nodes
    double *mn = nullptr, *mx = nullptr;   // [3][M]
    double *R3 = nullptr;                  // [4][M]: sum, x, y, z
    double *maxr = nullptr;                // [M]
    double *fs = nullptr;                  // [12][M]: F(3), P_ab(9)
    int32_t *first_child = nullptr, *next = nullptr, *leaf_start = nullptr, *count = nullptr;
    int32_t *child_cnt = nullptr;          // [M][8]
    int32_t *parents = nullptr, *parent_fc = nullptr;
    int32_t *flag = nullptr, *rank = nullptr;  // [M + 1]
    int32_t *fill = nullptr;               // [M]
    // particles
    double *p = nullptr;                   // [4][N]: x, y, z, r
    double *pf = nullptr;                  // [3][N]: forces of the last force walk
    int32_t *part_node = nullptr, *part_oct = nullptr, *leaf_idx = nullptr;
    int32_t *h_total = nullptr;            // pinned
    const dem_corr *corr = nullptr;        // periodic-image correction (borrowed), or none
};

namespace dem {

// Plain view of the tree passed to the kernels by value.
struct TreeDev {
    int cap, max_nodes, n, node_count, periodic;
    double L;
    double *mn, *mx, *R3, *maxr, *fs;
    int32_t *first_child, *next, *leaf_start, *count, *child_cnt, *parents, *parent_fc, *flag, *rank, *fill;
    double *p, *pf;
    int32_t *part_node, *part_oct, *leaf_idx;
    uint32_t *err;
};

static TreeDev view(const dem_tree *t) {
    TreeDev v;
    v.cap = t->cap;
    v.max_nodes = t->max_nodes;
    v.n = t->n;
    v.node_count = t->node_count;
    v.periodic = t->periodic;
    v.L = t->L;
    v.mn = t->mn;
    v.mx = t->mx;
    v.R3 = t->R3;
    v.maxr = t->maxr;
    v.fs = t->fs;
    v.first_child = t->first_child;
    v.next = t->next;
    v.leaf_start = t->leaf_start;
    v.count = t->count;
    v.child_cnt = t->child_cnt;
    v.parents = t->parents;
    v.parent_fc = t->parent_fc;
    v.flag = t->flag;
    v.rank = t->rank;
    v.fill = t->fill;
    v.p = t->p;
    v.pf = t->pf;
    v.part_node = t->part_node;
    v.part_oct = t->part_oct;
    v.leaf_idx = t->leaf_idx;
    v.err = t->ctx->d_err;
    return v;
}

__device__ __forceinline__ double node_size(const double *mn, const double *mx, int M, int k) {
    const double dx = mx[k] - mn[k], dy = mx[M + k] - mn[M + k], dz = mx[2 * M + k] - mn[2 * M + k];
    const double m = dx >= dy ? dx : dy;  // ti.max
    return m >= dz ? m : dz;
}

__device__ __forceinline__ void node_center(const double *mn, const double *mx, const double *R3, int M, int k,
                                            double &cx, double &cy, double &cz) {
    if (R3[k] > 0.0) {
        const double inv = 1.0 / R3[k];
        cx = R3[M + k] * inv;
        cy = R3[2 * M + k] * inv;
        cz = R3[3 * M + k] * inv;
    } else {
        cx = (mn[k] + mx[k]) * 0.5;
        cy = (mn[M + k] + mx[M + k]) * 0.5;
        cz = (mn[2 * M + k] + mx[2 * M + k]) * 0.5;
    }
}

// ---------------------------------------------------------------------------
// build
// ---------------------------------------------------------------------------
__global__ void tree_init_kernel(TreeDev t, int n, double L, const double *__restrict__ x,
                                 const double *__restrict__ y, const double *__restrict__ z,
                                 const double *__restrict__ r) {
    const int M = t.max_nodes, N = t.cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        t.p[i] = x[i];
        t.p[N + i] = y[i];
        t.p[2 * N + i] = z[i];
        t.p[3 * N + i] = r[i];
        t.part_node[i] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // _init_root_kernel :249-270
        for (int a = 0; a < 3; ++a) {
            t.mn[a * M] = 0.0;
            t.mx[a * M] = L;
        }
        t.first_child[0] = -1;
        t.next[0] = -1;
        t.leaf_start[0] = -1;
        t.count[0] = n;
        for (int a = 0; a < 4; ++a) t.R3[a * M] = 0.0;
        t.fs[0] = t.fs[M] = t.fs[2 * M] = 0.0;
    }
}

__global__ void zero_child_cnt_kernel(int32_t *child_cnt, int ls, int le) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < (le - ls) * 8; k += gridDim.x * blockDim.x)
        child_cnt[(size_t)ls * 8 + k] = 0;
}

// _level_assign_octants :284-306 (octree_node.py:84-95)
__global__ void assign_octants_kernel(TreeDev t, int n, int ls, int le) {
    const int M = t.max_nodes, N = t.cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int node = t.part_node[i];
        if (node >= ls && node < le) {
            const double cx = (t.mn[node] + t.mx[node]) * 0.5;
            const double cy = (t.mn[M + node] + t.mx[M + node]) * 0.5;
            const double cz = (t.mn[2 * M + node] + t.mx[2 * M + node]) * 0.5;
            int o = 0;
            if (t.p[i] >= cx) o |= 1;
            if (t.p[N + i] >= cy) o |= 2;
            if (t.p[2 * N + i] >= cz) o |= 4;
            t.part_oct[i] = o;
            atomicAdd(&t.child_cnt[(size_t)node * 8 + o], 1);
        }
    }
}

__global__ void subdivide_flags_kernel(TreeDev t, int ls, int le, int mpl) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < le - ls; k += gridDim.x * blockDim.x) {
        const int node = ls + k;
        t.flag[k] = (t.first_child[node] < 0 && t.count[node] > mpl) ? 1 : 0;
    }
}

// _level_subdivide_and_alloc :309-354 for the first `sub` candidates
__global__ void subdivide_kernel(TreeDev t, int ls, int le, int sub, int node_count, int parent_count) {
    const int M = t.max_nodes;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < le - ls; k += gridDim.x * blockDim.x) {
        if (!t.flag[k]) continue;
        const int q = t.rank[k];
        if (q >= sub) continue;
        const int node = ls + k;
        const int base = node_count + 8 * q;
        t.first_child[node] = base;
        t.parents[parent_count + q] = node;
        t.parent_fc[parent_count + q] = base;
        const double c[3] = {(t.mn[node] + t.mx[node]) * 0.5, (t.mn[M + node] + t.mx[M + node]) * 0.5,
                             (t.mn[2 * M + node] + t.mx[2 * M + node]) * 0.5};
        for (int o = 0; o < 8; ++o) {
            const int child = base + o;
            for (int a = 0; a < 3; ++a) {
                const bool up = (o >> a) & 1;
                t.mn[a * M + child] = up ? c[a] : t.mn[a * M + node];
                t.mx[a * M + child] = up ? t.mx[a * M + node] : c[a];
            }
            t.first_child[child] = -1;  // init_node, octree_node.py:117-154
            t.next[child] = -1;
            t.leaf_start[child] = -1;
            t.count[child] = t.child_cnt[(size_t)node * 8 + o];
            for (int a = 0; a < 4; ++a) t.R3[a * M + child] = 0.0;
            t.maxr[child] = 0.0;
            for (int a = 0; a < 12; ++a) t.fs[a * M + child] = 0.0;
        }
    }
}

// _level_scatter :357-366
__global__ void level_scatter_kernel(TreeDev t, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int node = t.part_node[i];
        if (node >= 0 && t.first_child[node] >= 0) t.part_node[i] = t.first_child[node] + t.part_oct[i];
    }
}

__global__ void leaf_flags_kernel(TreeDev t, int nc) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
        t.flag[k] = (t.first_child[k] < 0 && t.count[k] > 0) ? t.count[k] : 0;
        t.fill[k] = 0;
    }
}

// _finalize_leaves_alloc :371-385 (slots in node order)
__global__ void leaf_start_kernel(TreeDev t, int nc) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x)
        if (t.first_child[k] < 0 && t.count[k] > 0) t.leaf_start[k] = t.rank[k];
}

// _finalize_leaves_scatter :388-397
__global__ void leaf_scatter_kernel(TreeDev t, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int node = t.part_node[i];
        if (node >= 0 && t.first_child[node] < 0) {
            const int l0 = t.leaf_start[node];
            if (l0 >= 0) t.leaf_idx[l0 + atomicAdd(&t.fill[node], 1)] = i;
        }
    }
}

// particles of a leaf in ascending index order (the reference fills leaves serially)
__global__ void leaf_sort_kernel(TreeDev t, int nc) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
        if (!(t.first_child[k] < 0 && t.count[k] > 1 && t.leaf_start[k] >= 0)) continue;
        int32_t *a = t.leaf_idx + t.leaf_start[k];
        const int c = t.count[k];
        for (int u = 1; u < c; ++u) {
            const int32_t v = a[u];
            int w = u - 1;
            while (w >= 0 && a[w] > v) {
                a[w + 1] = a[w];
                --w;
            }
            a[w + 1] = v;
        }
    }
}

// _build_next_pointers_pass1 :400-415
__global__ void next_pass1_kernel(TreeDev t, int a, int b) {
    for (int i = a + blockIdx.x * blockDim.x + threadIdx.x; i < b; i += gridDim.x * blockDim.x) {
        const int parent = t.parents[i], base = t.parent_fc[i];
        const int pn = t.next[parent];
        for (int o = 0; o < 8; ++o) t.next[base + o] = (o == 7) ? pn : base + o + 1;
    }
}

// _build_next_pointers_pass2 :418-446
__global__ void next_pass2_kernel(TreeDev t, int a, int b) {
    for (int i = a + blockIdx.x * blockDim.x + threadIdx.x; i < b; i += gridDim.x * blockDim.x) {
        const int parent = t.parents[i], base = t.parent_fc[i];
        if (t.count[parent] == 0) {
            t.first_child[parent] = t.next[parent];
            continue;
        }
        int first = -1, last = -1;
        for (int j = 0; j < 8; ++j) {
            const int c = base + j;
            if (t.count[c] > 0) {
                if (first < 0) {
                    first = last = c;
                } else {
                    t.next[last] = c;
                    last = c;
                }
            }
        }
        if (last >= 0) {
            t.next[last] = t.next[parent];
            t.first_child[parent] = first;
        }
    }
}

// _init_leaf_r3 :470-511
__global__ void leaf_r3_kernel(TreeDev t, int nc) {
    const int M = t.max_nodes, N = t.cap;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
        double s = 0, wx = 0, wy = 0, wz = 0, mr = 0;
        if (t.first_child[k] < 0 && t.count[k] > 0 && t.leaf_start[k] >= 0) {
            const int l0 = t.leaf_start[k], c = t.count[k];
            for (int q = 0; q < c; ++q) {
                const int i = t.leaf_idx[l0 + q];
                if (i >= 0) {
                    const double ri = t.p[3 * N + i];
                    const double r3 = ipow3(ri);
                    s += r3;
                    wx += t.p[i] * r3;
                    wy += t.p[N + i] * r3;
                    wz += t.p[2 * N + i] * r3;
                    if (ri > mr) mr = ri;
                }
            }
        }
        t.R3[k] = s;
        t.R3[M + k] = wx;
        t.R3[2 * M + k] = wy;
        t.R3[3 * M + k] = wz;
        t.maxr[k] = mr;
        t.fs[k] = t.fs[M + k] = t.fs[2 * M + k] = 0.0;
    }
}

// _sweep_r3_level :514-542
__global__ void sweep_r3_kernel(TreeDev t, int a, int b) {
    const int M = t.max_nodes;
    for (int i = a + blockIdx.x * blockDim.x + threadIdx.x; i < b; i += gridDim.x * blockDim.x) {
        const int parent = t.parents[i], base = t.parent_fc[i];
        double s = 0, wx = 0, wy = 0, wz = 0, mr = 0;
        for (int j = 0; j < 8; ++j) {
            const int c = base + j;
            if (t.count[c] > 0) {
                s += t.R3[c];
                wx += t.R3[M + c];
                wy += t.R3[2 * M + c];
                wz += t.R3[3 * M + c];
                if (t.maxr[c] > mr) mr = t.maxr[c];
            }
        }
        t.R3[parent] = s;
        t.R3[M + parent] = wx;
        t.R3[2 * M + parent] = wy;
        t.R3[3 * M + parent] = wz;
        t.maxr[parent] = mr;
    }
}

// _init_leaf_forces(_from_fields) :556-627, :696-766
__global__ void leaf_forces_kernel(TreeDev t, int nc, const double *__restrict__ fx, const double *__restrict__ fy,
                                   const double *__restrict__ fz) {
    const int M = t.max_nodes, N = t.cap;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
        double s[3] = {0, 0, 0}, P[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (t.first_child[k] < 0 && t.count[k] > 0 && t.leaf_start[k] >= 0) {
            const int l0 = t.leaf_start[k], c = t.count[k];
            for (int q = 0; q < c; ++q) {
                const int i = t.leaf_idx[l0 + q];
                if (i >= 0) {
                    const double f[3] = {fx[i], fy[i], fz[i]};
                    const double xx[3] = {t.p[i], t.p[N + i], t.p[2 * N + i]};
                    s[0] += f[0];
                    s[1] += f[1];
                    s[2] += f[2];
                    for (int u = 0; u < 3; ++u)
                        for (int v = 0; v < 3; ++v) P[3 * u + v] += xx[u] * f[v];
                }
            }
        }
        for (int u = 0; u < 3; ++u) t.fs[u * M + k] = s[u];
        for (int u = 0; u < 9; ++u) t.fs[(3 + u) * M + k] = P[u];
    }
}

// _sweep_forces_level :629-672
__global__ void sweep_forces_kernel(TreeDev t, int a, int b) {
    const int M = t.max_nodes;
    for (int i = a + blockIdx.x * blockDim.x + threadIdx.x; i < b; i += gridDim.x * blockDim.x) {
        const int parent = t.parents[i], base = t.parent_fc[i];
        double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < 8; ++j) {
            const int c = base + j;
            if (t.count[c] > 0)
                for (int u = 0; u < 12; ++u) acc[u] += t.fs[u * M + c];
        }
        for (int u = 0; u < 12; ++u) t.fs[u * M + parent] = acc[u];
    }
}

// ---------------------------------------------------------------------------
// walks
// ---------------------------------------------------------------------------
// _compute_forces_kernel :783-894
template <bool PER>
__global__ void __launch_bounds__(128) force_walk_kernel(TreeDev t, double m_const, double theta_sq,
                                                         double *__restrict__ fx, double *__restrict__ fy,
                                                         double *__restrict__ fz) {
    const int M = t.max_nodes, N = t.cap, n = t.n;
    const double L = t.L, halfL = 0.5 * t.L;
    // targets in leaf-slot order (a permutation of all n particles: every particle ends in a leaf), so
    // the lanes of a warp walk neighbouring targets along nearly the same path; each target's sums
    // are its own thread's, in the reference's order, whatever order the targets are taken in
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        const int i = t.leaf_idx[slot];
        const double xi = t.p[i], yi = t.p[N + i], zi = t.p[2 * N + i], ri = t.p[3 * N + i];
        const double ri3 = ipow3(ri);
        double Fx = 0, Fy = 0, Fz = 0;
        int node = 0;
        int steps = 0;  // every node is visited at most once; more means broken links
        while (node >= 0) {
            if (++steps > t.node_count + 1) {
                raise_device_error(t.err, DEM_DEVERR_NODE_OVERFLOW);
                break;
            }
            const int cnt = t.count[node];
            if (cnt == 0 || t.R3[node] < 1e-30) {
                node = t.next[node];
                continue;
            }
            if (t.first_child[node] < 0) {
                const int l0 = t.leaf_start[node];
                for (int k = 0; k < cnt; ++k) {
                    const int j = t.leaf_idx[l0 + k];
                    if (j >= 0 && j != i) {
                        double dx = t.p[j] - xi, dy = t.p[N + j] - yi, dz = t.p[2 * N + j] - zi;
                        if (PER) {
                            dx = mic64(dx, L, halfL);
                            dy = mic64(dy, L, halfL);
                            dz = mic64(dz, L, halfL);
                        }
                        const double r_sq = dx * dx + dy * dy + dz * dz;
                        const double rj = t.p[3 * N + j];
                        const double r_sum = ri + rj;
                        if (r_sq >= r_sum * r_sum) {
                            const double rr = sqrt(r_sq);
                            const double r7 = r_sq * r_sq * r_sq * rr;
                            const double factor = m_const * ri3 * ipow3(rj) / r7;
                            const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
                            const double ang = 4.0 * dz2 - dx2 - dy2;
                            Fx += factor * dx * ang;
                            Fy += factor * dy * ang;
                            Fz += factor * dz * (2.0 * dz2 - 3.0 * dx2 - 3.0 * dy2);
                        }
                    }
                }
                node = t.next[node];
                continue;
            }
            const double s = node_size(t.mn, t.mx, M, node);
            double cx, cy, cz;
            node_center(t.mn, t.mx, t.R3, M, node, cx, cy, cz);
            double dx = cx - xi, dy = cy - yi, dz = cz - zi;
            if (PER) {
                dx = mic64(dx, L, halfL);
                dy = mic64(dy, L, halfL);
                dz = mic64(dz, L, halfL);
            }
            const double D_sq = dx * dx + dy * dy + dz * dz;
            if (s * s < theta_sq * D_sq && D_sq > 0.0) {
                const double rr = sqrt(D_sq);
                const double r7 = D_sq * D_sq * D_sq * rr;
                const double factor = m_const * ri3 * t.R3[node] / r7;
                const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
                const double ang = 4.0 * dz2 - dx2 - dy2;
                Fx += factor * dx * ang;
                Fy += factor * dy * ang;
                Fz += factor * dz * (2.0 * dz2 - 3.0 * dx2 - 3.0 * dy2);
                node = t.next[node];
            } else {
                node = t.first_child[node];
            }
        }
        fx[i] = Fx;
        fy[i] = Fy;
        fz[i] = Fz;
        t.pf[i] = Fx;
        t.pf[N + i] = Fy;
        t.pf[2 * N + i] = Fz;
    }
}

// _compute_stokeslet_kernel :1000-1280 (stokes <= 0) and
// _compute_total_velocity_kernel :1326-1588 (stokes > 0); with CORR the
// periodic-image correction after every leaf pair (:1070-1131) and accepted
// node (:1171-1213), and the self term of the Stokeslet walk (:1271-1276).
template <bool PER, bool CORR>
__global__ void __launch_bounds__(128) velocity_walk_kernel(TreeDev t, const double *__restrict__ Fx_,
                                                            const double *__restrict__ Fy_,
                                                            const double *__restrict__ Fz_, double eta,
                                                            double theta_sq, double stokes, CorrDev corr,
                                                            double *__restrict__ vx, double *__restrict__ vy,
                                                            double *__restrict__ vz) {
    const int M = t.max_nodes, N = t.cap, n = t.n;
    const double L = t.L, halfL = 0.5 * t.L;
    // targets in leaf-slot order, as in force_walk_kernel
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        const int i = t.leaf_idx[slot];
        const double xi = t.p[i], yi = t.p[N + i], zi = t.p[2 * N + i], ri = t.p[3 * N + i];
        double ux = 0, uy = 0, uz = 0;
        if (stokes > 0) {
            const double inv_stokes_r = 1.0 / (stokes * ri);
            ux = t.pf[i] * inv_stokes_r;
            uy = t.pf[N + i] * inv_stokes_r;
            uz = t.pf[2 * N + i] * inv_stokes_r;
        }
        int node = 0;
        int steps = 0;
        while (node >= 0) {
            if (++steps > t.node_count + 1) {
                raise_device_error(t.err, DEM_DEVERR_NODE_OVERFLOW);
                break;
            }
            const int cnt = t.count[node];
            const double fsx = t.fs[node], fsy = t.fs[M + node], fsz = t.fs[2 * M + node];
            const double fs2 = fsx * fsx + fsy * fsy + fsz * fsz;
            if (cnt == 0 || fs2 < 1e-60) {
                node = t.next[node];
                continue;
            }
            if (t.first_child[node] < 0) {
                const int l0 = t.leaf_start[node];
                for (int k = 0; k < cnt; ++k) {
                    const int j = t.leaf_idx[l0 + k];
                    if (j >= 0 && j != i) {
                        double dx = xi - t.p[j], dy = yi - t.p[N + j], dz = zi - t.p[2 * N + j];
                        if (PER) {
                            dx = mic64(dx, L, halfL);
                            dy = mic64(dy, L, halfL);
                            dz = mic64(dz, L, halfL);
                        }
                        const double r_sq = dx * dx + dy * dy + dz * dz;
                        const double r_sum = ri + t.p[3 * N + j];
                        if (r_sq >= r_sum * r_sum) {
                            const double rr = sqrt(r_sq);
                            const double inv_r = 1.0 / rr;
                            const double inv_r2 = inv_r * inv_r;
                            const double Fx = Fx_[j], Fy = Fy_[j], Fz = Fz_[j];
                            const double dot = dx * Fx + dy * Fy + dz * Fz;
                            const double coeff = eta * inv_r;
                            ux += coeff * (Fx + dx * inv_r2 * dot);
                            uy += coeff * (Fy + dy * inv_r2 * dot);
                            uz += coeff * (Fz + dz * inv_r2 * dot);
                            if (CORR) corr_pair64(corr, dx, dy, dz, Fx, Fy, Fz, ux, uy, uz);
                        }
                    }
                }
                node = t.next[node];
                continue;
            }
            const double s = node_size(t.mn, t.mx, M, node);
            double cx, cy, cz;
            node_center(t.mn, t.mx, t.R3, M, node, cx, cy, cz);
            double dx = xi - cx, dy = yi - cy, dz = zi - cz;
            if (PER) {
                dx = mic64(dx, L, halfL);
                dy = mic64(dy, L, halfL);
                dz = mic64(dz, L, halfL);
            }
            const double D_sq = dx * dx + dy * dy + dz * dz;
            if (s * s < theta_sq * D_sq && D_sq > 0.0) {
                const double rr = sqrt(D_sq);
                const double inv_r = 1.0 / rr;
                const double inv_r2 = inv_r * inv_r;
                const double Fx = fsx, Fy = fsy, Fz = fsz;
                const double dot = dx * Fx + dy * Fy + dz * Fz;
                const double coeff = eta * inv_r;
                ux += coeff * (Fx + dx * inv_r2 * dot);
                uy += coeff * (Fy + dy * inv_r2 * dot);
                uz += coeff * (Fz + dz * inv_r2 * dot);
                if (CORR) corr_pair64(corr, dx, dy, dz, Fx, Fy, Fz, ux, uy, uz);
                // dipole correction :1215-1265, R^3-weighted centre (same as get_center)
                const double cmx = cx, cmy = cy, cmz = cz;
                const double *P = t.fs + 3 * (size_t)M;
                const double Dxx = P[node] - cmx * Fx, Dxy = P[M + node] - cmx * Fy, Dxz = P[2 * M + node] - cmx * Fz;
                const double Dyx = P[3 * M + node] - cmy * Fx, Dyy = P[4 * M + node] - cmy * Fy,
                             Dyz = P[5 * M + node] - cmy * Fz;
                const double Dzx = P[6 * M + node] - cmz * Fx, Dzy = P[7 * M + node] - cmz * Fy,
                             Dzz = P[8 * M + node] - cmz * Fz;
                const double rx = dx, ry = dy, rz = dz;
                const double Ux = Dxx * rx + Dyx * ry + Dzx * rz;
                const double Uy = Dxy * rx + Dyy * ry + Dzy * rz;
                const double Uz = Dxz * rx + Dyz * ry + Dzz * rz;
                const double wx = Dxx * rx + Dxy * ry + Dxz * rz;
                const double wy = Dyx * rx + Dyy * ry + Dyz * rz;
                const double wz = Dzx * rx + Dzy * ry + Dzz * rz;
                const double s_tr = Dxx + Dyy + Dzz;
                const double q = rx * wx + ry * wy + rz * wz;
                const double inv_r3 = inv_r * inv_r2;
                const double inv_r5 = inv_r3 * inv_r2;
                ux += eta * (inv_r3 * (Ux - wx - s_tr * rx) + 3.0 * rx * q * inv_r5);
                uy += eta * (inv_r3 * (Uy - wy - s_tr * ry) + 3.0 * ry * q * inv_r5);
                uz += eta * (inv_r3 * (Uz - wz - s_tr * rz) + 3.0 * rz * q * inv_r5);
                node = t.next[node];
            } else {
                node = t.first_child[node];
            }
        }
        if (CORR && !(stokes > 0)) {  // self term, Stokeslet walk only
            ux += corr.g_self * Fx_[i];
            uy += corr.g_self * Fy_[i];
            uz += corr.g_self * Fz_[i];
        }
        vx[i] = ux;
        vy[i] = uy;
        vz[i] = uz;
    }
}

// TreeCollisionFrequency._count_collisions, pbm/collision_frequency/tree_collision_freq.py:62-135:
// every pair j > i with |MIC(x_j - x_i)|^2 <= (r_i + r_j)^2 adds 1 to matrix[b_i][b_j]
// and to matrix[b_j][b_i]; a node is skipped when the squared distance from x_i to
// its box exceeds (r_i + max radius in the node)^2, the box distance taken per
// axis as the gap to the nearer face and, when periodic, replaced by L - gap
// when the gap exceeds L/2 (:137-175), as the reference does.
template <bool PER>
__global__ void collision_walk_kernel(TreeDev t, const int32_t *__restrict__ bins, int nbins,
                                      unsigned int *__restrict__ matrix) {
    const int M = t.max_nodes, N = t.cap, n = t.n;
    const double L = t.L, halfL = 0.5 * t.L;
    // targets in leaf-slot order, as in force_walk_kernel (the counts are integers: any order)
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        const int i = t.leaf_idx[slot];
        const double xi = t.p[i], yi = t.p[N + i], zi = t.p[2 * N + i], ri = t.p[3 * N + i];
        const int bi = bins[i];
        int node = 0, steps = 0;
        while (node >= 0) {
            if (++steps > t.node_count + 1) {
                raise_device_error(t.err, DEM_DEVERR_NODE_OVERFLOW);
                break;
            }
            const int cnt = t.count[node];
            if (cnt == 0) {
                node = t.next[node];
                continue;
            }
            if (t.first_child[node] < 0) {
                const int l0 = t.leaf_start[node];
                for (int k = 0; k < cnt; ++k) {
                    const int j = t.leaf_idx[l0 + k];
                    if (j >= 0 && j > i) {
                        double dx = t.p[j] - xi, dy = t.p[N + j] - yi, dz = t.p[2 * N + j] - zi;
                        if (PER) {
                            dx = mic64(dx, L, halfL);
                            dy = mic64(dy, L, halfL);
                            dz = mic64(dz, L, halfL);
                        }
                        const double dist_sq = dx * dx + dy * dy + dz * dz;
                        const double contact = ri + t.p[3 * N + j];
                        if (dist_sq <= contact * contact) {
                            const int bj = bins[j];
                            atomicAdd(&matrix[bi * nbins + bj], 1u);
                            atomicAdd(&matrix[bj * nbins + bi], 1u);
                        }
                    }
                }
                node = t.next[node];
                continue;
            }
            const double max_contact = ri + t.maxr[node];
            double g[3];
            const double p3[3] = {xi, yi, zi};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const double lo = t.mn[a * (size_t)M + node], hi = t.mx[a * (size_t)M + node];
                double d = 0.0;
                if (p3[a] < lo)
                    d = lo - p3[a];
                else if (p3[a] > hi)
                    d = p3[a] - hi;
                if (PER && L > 0.0 && d > halfL) d = L - d;
                g[a] = d;
            }
            const double min_dist_sq = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
            node = min_dist_sq > max_contact * max_contact ? t.next[node] : t.first_child[node];
        }
    }
}

__global__ void copy_nodes_kernel(TreeDev t, int nc, int32_t *count, int32_t *first_child, int32_t *next,
                                  int32_t *leaf_start, double *r3, double *fs) {
    const int M = t.max_nodes;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
        if (count) count[k] = t.count[k];
        if (first_child) first_child[k] = t.first_child[k];
        if (next) next[k] = t.next[k];
        if (leaf_start) leaf_start[k] = t.leaf_start[k];
        if (r3)
            for (int a = 0; a < 4; ++a) r3[4 * (size_t)k + a] = t.R3[a * M + k];
        if (fs)
            for (int a = 0; a < 12; ++a) fs[12 * (size_t)k + a] = t.fs[a * M + k];
    }
}

static int grid_for(dem_ctx *ctx, int64_t work) { return (int)max(1LL, min((long long)ceil_div(work, 256), 16LL * ctx->sm_count)); }

}  // namespace dem

using namespace dem;

static int tree_free(dem_tree *t) {
    void *ptrs[] = {t->mn,       t->mx,   t->R3,       t->maxr,      t->fs,   t->first_child, t->next,
                    t->leaf_start, t->count, t->child_cnt, t->parents, t->parent_fc, t->flag, t->rank,
                    t->fill,     t->p,    t->pf,       t->part_node, t->part_oct, t->leaf_idx};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (t->h_total) cudaFreeHost(t->h_total);
    return DEM_OK;
}

extern "C" {

int dem_tree_create(dem_ctx *ctx, int capacity, int max_nodes, dem_tree **out) {
    if (!ctx || !out || capacity < 1 || max_nodes < 1) return DEM_E_INVALID;
    *out = nullptr;
    dem_tree *t = new dem_tree();
    t->ctx = ctx;
    t->device = ctx->device;
    t->cap = capacity;
    t->max_nodes = max_nodes;
    const size_t M = (size_t)max_nodes, N = (size_t)capacity;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaSuccess;
#define ALLOC(f, T, k) \
    if (e == cudaSuccess) e = cudaMalloc((void **)&t->f, sizeof(T) * (k))
    ALLOC(mn, double, 3 * M);
    ALLOC(mx, double, 3 * M);
    ALLOC(R3, double, 4 * M);
    ALLOC(maxr, double, M);
    ALLOC(fs, double, 12 * M);
    ALLOC(first_child, int32_t, M);
    ALLOC(next, int32_t, M);
    ALLOC(leaf_start, int32_t, M);
    ALLOC(count, int32_t, M);
    ALLOC(child_cnt, int32_t, 8 * M);
    ALLOC(parents, int32_t, M);
    ALLOC(parent_fc, int32_t, M);
    ALLOC(flag, int32_t, M + 1);
    ALLOC(rank, int32_t, M + 1);
    ALLOC(fill, int32_t, M);
    ALLOC(p, double, 4 * N);
    ALLOC(pf, double, 3 * N);
    ALLOC(part_node, int32_t, N);
    ALLOC(part_oct, int32_t, N);
    ALLOC(leaf_idx, int32_t, N);
#undef ALLOC
    if (e == cudaSuccess) e = cudaMallocHost((void **)&t->h_total, sizeof(int32_t) * 2);
    if (e != cudaSuccess) {
        tree_free(t);
        delete t;
        return dem_set_error(ctx, DEM_E_CUDA, std::string("tree allocation: ") + cudaGetErrorString(e));
    }
    *out = t;
    return DEM_OK;
}

void dem_tree_destroy(dem_tree *t) {
    if (!t) return;
    cudaSetDevice(t->device);
    tree_free(t);
    delete t;
}

int dem_tree_build(dem_tree *t, int n, const double *x, const double *y, const double *z, const double *r, double L,
                   int periodic, int mpl, void *stream) {
    if (!t) return DEM_E_INVALID;
    dem_ctx *ctx = t->ctx;
    if (n < 0) return dem_set_error(ctx, DEM_E_INVALID, "n must be >= 0");
    if (n > t->cap)
        return dem_set_error(ctx, DEM_E_CAPACITY, "Number of particles (" + std::to_string(n) +
                                                      ") exceeds allocated capacity (" + std::to_string(t->cap) + ")");
    cudaSetDevice(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    t->n = n;
    t->L = L;
    t->periodic = periodic ? 1 : 0;
    t->node_count = 1;
    t->parent_count = 0;
    t->pool_exhausted = 0;
    t->level_off.clear();
    dem_prof_begin(ctx, "tree_build", s);
    tree_init_kernel<<<grid_for(ctx, max(n, 1)), 256, 0, counted(s)>>>(view(t), n, L, x, y, z, r);
    int ls = 0, le = 1;
    for (int level = 0; level < 40; ++level) {
        const int pc_before = t->parent_count;
        const int width = le - ls;
        zero_child_cnt_kernel<<<grid_for(ctx, 8LL * width), 256, 0, counted(s)>>>(t->child_cnt, ls, le);
        assign_octants_kernel<<<grid_for(ctx, max(n, 1)), 256, 0, counted(s)>>>(view(t), n, ls, le);
        subdivide_flags_kernel<<<grid_for(ctx, width), 256, 0, counted(s)>>>(view(t), ls, le, mpl);
        int rc = exclusive_scan<int32_t, int32_t>(ctx, t->flag, t->rank, width, s);
        if (rc) return rc;
        rc = dem_check_cuda(ctx, cudaMemcpyAsync(t->h_total, t->rank + width, sizeof(int32_t), cudaMemcpyDeviceToHost, s),
                            "tree build");
        if (!rc) rc = dem_check_cuda(ctx, cudaStreamSynchronize(s), "tree build");
        if (rc) return rc;
        const int total = t->h_total[0];
        const int room = (t->max_nodes - t->node_count) / 8;
        const int sub = total < room ? total : (room > 0 ? room : 0);
        if (sub < total) t->pool_exhausted = 1;
        if (sub > 0) {
            subdivide_kernel<<<grid_for(ctx, width), 256, 0, counted(s)>>>(view(t), ls, le, sub, t->node_count, t->parent_count);
            t->node_count += 8 * sub;
            t->parent_count += sub;
        }
        level_scatter_kernel<<<grid_for(ctx, max(n, 1)), 256, 0, counted(s)>>>(view(t), n);
        ls = le;
        le = t->node_count;
        if (t->parent_count > pc_before) t->level_off.push_back(pc_before);
        if (sub == 0) break;
    }
    const int nc = t->node_count;
    leaf_flags_kernel<<<grid_for(ctx, nc), 256, 0, counted(s)>>>(view(t), nc);
    int rc = exclusive_scan<int32_t, int32_t>(ctx, t->flag, t->rank, nc, s);
    if (rc) return rc;
    leaf_start_kernel<<<grid_for(ctx, nc), 256, 0, counted(s)>>>(view(t), nc);
    leaf_scatter_kernel<<<grid_for(ctx, max(n, 1)), 256, 0, counted(s)>>>(view(t), n);
    leaf_sort_kernel<<<grid_for(ctx, nc), 256, 0, counted(s)>>>(view(t), nc);
    const int nl = (int)t->level_off.size();
    auto lev_end = [&](int l) { return l + 1 < nl ? t->level_off[l + 1] : t->parent_count; };
    for (int l = 0; l < nl; ++l)
        next_pass1_kernel<<<grid_for(ctx, lev_end(l) - t->level_off[l]), 256, 0, counted(s)>>>(view(t), t->level_off[l], lev_end(l));
    for (int l = 0; l < nl; ++l)
        next_pass2_kernel<<<grid_for(ctx, lev_end(l) - t->level_off[l]), 256, 0, counted(s)>>>(view(t), t->level_off[l], lev_end(l));
    leaf_r3_kernel<<<grid_for(ctx, nc), 256, 0, counted(s)>>>(view(t), nc);
    for (int l = nl - 1; l >= 0; --l)
        sweep_r3_kernel<<<grid_for(ctx, lev_end(l) - t->level_off[l]), 256, 0, counted(s)>>>(view(t), t->level_off[l], lev_end(l));
    rc = dem_check_cuda(ctx, cudaMemcpyAsync(t->h_total + 1, t->rank + nc, sizeof(int32_t), cudaMemcpyDeviceToHost, s),
                        "tree build");
    if (!rc) rc = dem_check_cuda(ctx, cudaStreamSynchronize(s), "tree build");
    if (rc) return rc;
    t->leaf_slot_count = t->h_total[1];
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "tree build");
}

int dem_tree_forces(dem_tree *t, double m_const, double theta_sq, double *fx, double *fy, double *fz, void *stream) {
    if (!t || !fx || !fy || !fz) return DEM_E_INVALID;
    if (t->n == 0) return DEM_OK;
    cudaStream_t s = (cudaStream_t)stream;
    dem_prof_begin(t->ctx, "tree_force_walk", s);
    const int grid = ceil_div(t->n, 128);
    if (t->periodic)
        force_walk_kernel<true><<<grid, 128, 0, counted(s)>>>(view(t), m_const, theta_sq, fx, fy, fz);
    else
        force_walk_kernel<false><<<grid, 128, 0, counted(s)>>>(view(t), m_const, theta_sq, fx, fy, fz);
    dem_prof_end(t->ctx, s);
    return dem_check_launch(t->ctx, "tree force walk");
}

int dem_tree_propagate_forces(dem_tree *t, const double *fx, const double *fy, const double *fz, void *stream) {
    if (!t) return DEM_E_INVALID;
    dem_ctx *ctx = t->ctx;
    cudaStream_t s = (cudaStream_t)stream;
    const int N = t->cap, nc = t->node_count;
    if (!fx) {
        fx = t->pf;
        fy = t->pf + N;
        fz = t->pf + 2 * (size_t)N;
    }
    leaf_forces_kernel<<<grid_for(ctx, nc), 256, 0, counted(s)>>>(view(t), nc, fx, fy, fz);
    const int nl = (int)t->level_off.size();
    for (int l = nl - 1; l >= 0; --l) {
        const int a = t->level_off[l], b = l + 1 < nl ? t->level_off[l + 1] : t->parent_count;
        sweep_forces_kernel<<<grid_for(ctx, b - a), 256, 0, counted(s)>>>(view(t), a, b);
    }
    return dem_check_launch(ctx, "tree propagate forces");
}

int dem_tree_velocity(dem_tree *t, const double *fx, const double *fy, const double *fz, double eta_const,
                      double theta_sq, double stokes_factor, double *vx, double *vy, double *vz, void *stream) {
    if (!t || !vx || !vy || !vz) return DEM_E_INVALID;
    if (t->n == 0) return DEM_OK;
    const int N = t->cap;
    if (!fx) {
        fx = t->pf;
        fy = t->pf + N;
        fz = t->pf + 2 * (size_t)N;
    }
    cudaStream_t s = (cudaStream_t)stream;
    dem_prof_begin(t->ctx, "tree_velocity_walk", s);
    const int grid = ceil_div(t->n, 128);
    const TreeDev tv = view(t);
    if (t->corr) {
        const CorrDev cv = corr_view(t->corr);
        if (t->periodic)
            velocity_walk_kernel<true, true><<<grid, 128, 0, counted(s)>>>(tv, fx, fy, fz, eta_const, theta_sq,
                                                                           stokes_factor, cv, vx, vy, vz);
        else
            velocity_walk_kernel<false, true><<<grid, 128, 0, counted(s)>>>(tv, fx, fy, fz, eta_const, theta_sq,
                                                                            stokes_factor, cv, vx, vy, vz);
    } else {
        const CorrDev none{};
        if (t->periodic)
            velocity_walk_kernel<true, false><<<grid, 128, 0, counted(s)>>>(tv, fx, fy, fz, eta_const, theta_sq,
                                                                            stokes_factor, none, vx, vy, vz);
        else
            velocity_walk_kernel<false, false><<<grid, 128, 0, counted(s)>>>(tv, fx, fy, fz, eta_const, theta_sq,
                                                                             stokes_factor, none, vx, vy, vz);
    }
    dem_prof_end(t->ctx, s);
    return dem_check_launch(t->ctx, "tree velocity walk");
}

int dem_tree_set_correction(dem_tree *t, const dem_corr *corr) {
    if (!t) return DEM_E_INVALID;
    if (corr && corr->ctx && corr->ctx->device != t->device)
        return dem_set_error(t->ctx, DEM_E_INVALID, "correction grid lives on another device");
    t->corr = corr;
    return DEM_OK;
}

int dem_tree_stats(const dem_tree *t, int64_t *out) {
    if (!t || !out) return DEM_E_INVALID;
    out[0] = t->node_count;
    out[1] = t->parent_count;
    out[2] = t->leaf_slot_count;
    out[3] = t->max_nodes;
    out[4] = (int64_t)t->level_off.size();
    out[5] = t->n;
    out[6] = t->pool_exhausted;
    out[7] = t->cap;
    return DEM_OK;
}

int dem_tree_nodes(dem_tree *t, int32_t *count, int32_t *first_child, int32_t *next, int32_t *leaf_start, double *r3,
                   double *fs, void *stream) {
    if (!t) return DEM_E_INVALID;
    const int nc = t->node_count;
    copy_nodes_kernel<<<grid_for(t->ctx, nc), 256, 0, counted((cudaStream_t)stream)>>>(view(t), nc, count, first_child, next,
                                                                             leaf_start, r3, fs);
    return dem_check_launch(t->ctx, "tree nodes");
}

int dem_tree_collision_matrix(dem_tree *t, const int32_t *bins, int nbins, uint32_t *matrix, void *stream) {
    if (!t || nbins < 1 || !matrix || (t->n > 0 && !bins)) return DEM_E_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = dem_check_cuda(t->ctx, cudaMemsetAsync(matrix, 0, sizeof(uint32_t) * nbins * nbins, s), "memset");
    if (rc || t->n == 0) return rc;
    const int grid = ceil_div(t->n, 128);
    dem_prof_begin(t->ctx, "tree_collision_walk", s);
    if (t->periodic)
        collision_walk_kernel<true><<<grid, 128, 0, counted(s)>>>(view(t), bins, nbins, matrix);
    else
        collision_walk_kernel<false><<<grid, 128, 0, counted(s)>>>(view(t), bins, nbins, matrix);
    dem_prof_end(t->ctx, s);
    return dem_check_launch(t->ctx, "tree collision walk");
}

int dem_tree_leaf_indices(dem_tree *t, int32_t *out, void *stream) {
    if (!t || !out) return DEM_E_INVALID;
    if (t->n == 0) return DEM_OK;
    return dem_check_cuda(t->ctx,
                          cudaMemcpyAsync(out, t->leaf_idx, sizeof(int32_t) * t->n, cudaMemcpyDeviceToDevice,
                                          (cudaStream_t)stream),
                          "leaf indices");
}

}  // extern "C"
