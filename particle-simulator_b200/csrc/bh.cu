// bh.cu -- Barnes-Hut octree from Morton keys, warp-cooperative FP32 walks.
//
// The reference's flat octree (dem/octree/flat_tree.py, octree_node.py) is
// built by serial subdivision and walked per particle in FP64 (tree.cu keeps
// that form for parity).  This file is the fast form of the same method:
//
//   build   30-bit Morton keys (10 bits per axis) of the positions in the root
//           cube -> stable LSD radix sort (8-bit digits, warp-ranked scatter)
//           -> particles gathered into key order -> octree level by level from
//           key prefixes: a node is a run of keys sharing 3*level leading
//           bits, split into its non-empty octants while it holds more than
//           `leaf_size` droplets (and level < 10); nodes are contiguous runs
//           of the sorted arrays, children stored consecutively.
//           Algorithmic bytes of the build: 156 N + 140 M (N droplets, M nodes):
//           positions read and key written (28 B), four radix passes over
//           (key, index) (64 B), position and radius gathered into key order
//           (64 B), the node records written.
//   nodes   R^3 sum and R^3-weighted centre (flat_tree.py:544-554,
//           octree_node.py:98-114), side = root side / 2^level, and the
//           R^3-weighted second moment Q of the node about that centre; after the force
//           walk, sum F and the dipole D = sum (x - c) F^T (= P - c F^T of
//           flat_tree.py:556-777).  Both bottom up, one level per launch: a leaf
//           sums its droplets, an inner node its children's FP64 sums moved to
//           its own reference point (first droplet, resp. centre).
//   walks   one warp per 64 consecutive sorted targets, two per lane, their
//           terms evaluated in packed FP32x2 (bh_walk2_kernel; with the
//           periodic-image correction, one target per lane: bh_walk_kernel); the
//           warp shares a shared-memory stack and opens a node when any of its
//           targets fails the reference's acceptance test s^2 < theta^2 D^2
//           (flat_tree.py:871), so every target sees a tree cut at least as fine
//           as its own; in a
//           periodic box a node of level < window_level is also opened
//           unless its whole cell lies in the target's minimum-image window
//           (|D_axis| + s < L/2), where all its droplets take the image of its
//           centre (the reference evaluates such a node at its centre's image).
//           Accepted nodes: monopole force (:873-884) plus its quadrupole
//           correction / Stokeslet + dipole correction (:1215-1265); leaves:
//           exact pair terms with the
//           contact cut r^2 >= (r_i + r_j)^2 (:835).  Separations are taken in
//           FP64 from FP64 positions (minimum image), the terms in FP32.
//
// Quadrupole correction of the node force.  The pair force is f(d) = P(d)/|d|^7
// = grad(phi)/3 with phi(d) = |d|^-3 - 3 dz^2 |d|^-5.  About the R^3-weighted
// centre c the first-order term of sum_j r_j^3 f(D + delta_j) vanishes, so the
// next term is (1/6) Q_ab d_a d_b d_c phi(D) with Q = sum_j r_j^3 delta_j delta_j^T;
// with x = D, S_abc = delta_ab x_c + delta_ac x_b + delta_bc x_a, the third
// derivatives of |d|^-n are n(n+2) [S_abc r^-(n+4) - (n+4) x_a x_b x_c r^-(n+6)]
// and those of dz^2 |d|^-5 follow from the product rule; contracted with Q they
// give the closed form of quad_force below.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "corr.cuh"
#include "mixed_common.cuh"
#include "morton.cuh"
#include "scan.cuh"

namespace dem {

constexpr int RS_T = 256, RS_ITEMS = 8, RS_TILE = RS_T * RS_ITEMS;
constexpr int BH_T = 128;     // threads per walk CTA (4 warps)
constexpr int BH_STACK = 96;  // stack entries per warp (depth <= 10, <= 8 children per node)
// resident CTAs per SM the two-target walks are compiled for (5: 94-96 registers, none spilled; 0.4 %
// faster at N = 2^20 than 4 CTAs with 107-108 registers)
#ifndef BH_WALK2_CTAS_FORCE
#define BH_WALK2_CTAS_FORCE 5
#endif
#ifndef BH_WALK2_CTAS_VEL
#define BH_WALK2_CTAS_VEL 5
#endif
constexpr int BH_MAX_LEVEL = 10;
// meta.w = level | flags: the walks pass over a flagged node without a term (empty, or the reference's
// skip tests: R^3 sum < 1e-30 m^3, flat_tree.py:861; |F sum|^2 < 1e-60 N^2, flat_tree.py:1155)
constexpr int BH_LEVEL_MASK = 0xff;
constexpr int BH_SKIP_FORCE = 0x100;
constexpr int BH_SKIP_VEL = 0x200;

struct BhNodes {
    int *start, *count, *first_child, *nchild, *level;
    double *cx, *cy, *cz;  // R^3-weighted centre
    double *mom;           // [22][M] FP64 moment sums of the bottom-up pass (node_r3_up / node_force_up)
    float4 *cs;            // walk copy: centre relative to the root cube origin / ell, and side / ell
    int4 *meta;            // walk copy: count, nchild, first child (a leaf: first droplet), level | skip flags
    // walk records, one 16-byte-aligned group per node so that a visit issues vector loads:
    float4 *qr;  // [M][2] second moment Q = sum r^3 (x - c)(x - c)^T and R^3 sum:
                 //        (Qxx, Qxy, Qxz, Qyy), (Qyz, Qzz, R^3, 0)
    float4 *fd;  // [M][3] force sum and dipole D_ab = sum (x_a - c_a) F_b (row a, column b), as its
                 // symmetric part S = (D + D^T) / 2 and antisymmetric part A = D^T - D:
                 //        (Fx, Fy, Fz, Sxx), (Syy, Szz, 2 Sxy, 2 Sxz), (2 Syz, A01, A02, A12)
                 // (the walk's dipole term needs A e, e.S e and tr S only)
};

}  // namespace dem

using namespace dem;

struct dem_bh {
    dem_ctx *ctx = nullptr;
    int capacity = 0, max_nodes = 0;
    int n = 0, node_count = 0, leaf_size = 16, periodic = 0, nlevels = 0;
    int window_level = 0;  // see dem_bh_set_window (0: the reference's acceptance rule)
    double L = 1.0;
    uint32_t *keys[2] = {nullptr, nullptr};
    int32_t *idx[2] = {nullptr, nullptr};
    int32_t *hist = nullptr;
    double *ps = nullptr;       // [4][capacity] sorted x, y, z, r
    double *fsort = nullptr;    // [3][capacity] forces in sorted order
    float4 *loff = nullptr;     // [capacity] (x - c_leaf, y - c_leaf, z - c_leaf, r) / ell per sorted droplet
    float4 *fs32 = nullptr;     // [capacity] sorted forces scaled by 2^-q (velocity walk)
    int32_t *bounds = nullptr;  // [9][max_nodes] child split points of the current level
    long long *bbox = nullptr;  // [6] min/max of an open box (order-preserving integers)
    double *geom = nullptr;     // [4] root cube origin x, y, z and side
    unsigned long long *counters = nullptr;       // [2] pair and node terms of the last walk
    unsigned long long *scales = nullptr;         // [2] max r, max |F| (bit patterns)
    int32_t *scan_in = nullptr, *coff = nullptr;  // [max_nodes + 1] children per node of a level, offsets
    BhNodes nd{};
    std::vector<int> level_off;
    const dem_corr *corr = nullptr;  // periodic-image correction of the velocity walk (borrowed), or none
};

namespace {

__device__ __forceinline__ uint32_t spread10(uint32_t v) {  // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t compact10(uint32_t v) {  // inverse of spread10
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030C30C3u;
    v = (v | (v >> 4)) & 0x0300F00Fu;
    v = (v | (v >> 8)) & 0x030000FFu;
    v = (v | (v >> 16)) & 0x3ffu;
    return v;
}

__device__ __forceinline__ uint32_t cell10(double p, double o, double inv_side) {
    const double t = (p - o) * inv_side * 1024.0;
    int c = (int)floor(t);
    c = c < 0 ? 0 : (c > 1023 ? 1023 : c);
    return (uint32_t)c;
}

// Doubles as order-preserving signed integers (for atomicMin / atomicMax).
__device__ __forceinline__ long long ord_of(double v) {
    const long long b = __double_as_longlong(v);
    return b >= 0 ? b : (long long)(0x8000000000000000ULL - (unsigned long long)b);
}
__device__ __forceinline__ double of_ord(long long m) {
    return __longlong_as_double(m >= 0 ? m : (long long)(0x8000000000000000ULL - (unsigned long long)m));
}

__global__ void bbox_init_kernel(long long *bb) {
    if (threadIdx.x < 3)
        bb[threadIdx.x] = ord_of(1e300);
    else if (threadIdx.x < 6)
        bb[threadIdx.x] = ord_of(-1e300);
}

__global__ void bbox_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, long long *bb) {
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v[3] = {x[i], y[i], z[i]};
        for (int c = 0; c < 3; ++c) {
            mn[c] = fmin(mn[c], v[c]);
            mx[c] = fmax(mx[c], v[c]);
        }
    }
    for (int c = 0; c < 3; ++c) {
        for (int o = 16; o; o >>= 1) {
            mn[c] = fmin(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
            mx[c] = fmax(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int c = 0; c < 3; ++c) {
            atomicMin(&bb[c], ord_of(mn[c]));
            atomicMax(&bb[3 + c], ord_of(mx[c]));
        }
    }
}

// Root cube: [0, L)^3 for a periodic box, else the bounding cube of the droplets.
__global__ void geom_kernel(int periodic, double L, const long long *bb, double *geom) {
    if (threadIdx.x != 0) return;
    if (periodic) {
        geom[0] = geom[1] = geom[2] = 0.0;
        geom[3] = L;
        return;
    }
    double side = 0.0;
    for (int c = 0; c < 3; ++c) {
        geom[c] = of_ord(bb[c]);
        side = fmax(side, of_ord(bb[3 + c]) - geom[c]);
    }
    geom[3] = side > 0.0 ? side * (1.0 + 1e-12) : 1.0;
}

__global__ void keys_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, const double *__restrict__ geom,
                            uint32_t *__restrict__ keys, int32_t *__restrict__ idx) {
    const double ox = geom[0], oy = geom[1], oz = geom[2], inv_side = 1.0 / geom[3];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t cx = cell10(x[i], ox, inv_side), cy = cell10(y[i], oy, inv_side),
                       cz = cell10(z[i], oz, inv_side);
        keys[i] = (spread10(cx) << 2) | (spread10(cy) << 1) | spread10(cz);
        idx[i] = i;
    }
}

// Per-tile digit histogram, digit-major: hist[d * tiles + tile].
__global__ void __launch_bounds__(RS_T) rs_hist_kernel(int n, const uint32_t *__restrict__ keys, int shift,
                                                       int tiles, int32_t *__restrict__ hist) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; ++k) {
        const int i = base + k * RS_T + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: warp w ranks items [w * 256, (w + 1) * 256) of the tile in
// order, 32 at a time, grouping equal digits with match.any.
__global__ void __launch_bounds__(RS_T) rs_scatter_kernel(int n, const uint32_t *__restrict__ kin,
                                                          const int32_t *__restrict__ vin, uint32_t *__restrict__ kout,
                                                          int32_t *__restrict__ vout, int shift, int tiles,
                                                          const int32_t *__restrict__ off) {
    constexpr int W = RS_T / 32;
    __shared__ int cnt[W][256];
    __shared__ int run[W][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < W * 256; d += RS_T) (&cnt[0][0])[d] = 0;
    __syncthreads();
    const int base = blockIdx.x * RS_TILE + w * (32 * RS_ITEMS);
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < RS_ITEMS; ++r) {
        const int i = base + r * 32 + lane;
        const bool valid = i < n;
        const int d = valid ? (int)((kin[i] >> shift) & 255u) : 256 + lane;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (valid && (peers & lt) == 0) cnt[w][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        const int d = threadIdx.x;  // RS_T == 256 digits
        int acc = off[d * tiles + blockIdx.x];
        for (int ww = 0; ww < W; ++ww) {
            run[ww][d] = acc;
            acc += cnt[ww][d];
        }
    }
    __syncthreads();
    for (int r = 0; r < RS_ITEMS; ++r) {
        const int i = base + r * 32 + lane;
        const bool valid = i < n;
        const uint32_t key = valid ? kin[i] : 0u;
        const int d = valid ? (int)((key >> shift) & 255u) : 256 + lane;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        int pos = 0;
        if (valid) pos = run[w][d] + __popc(peers & lt);
        __syncwarp();
        if (valid) {
            kout[pos] = key;
            vout[pos] = vin[i];
            if ((peers & lt) == 0) run[w][d] += __popc(peers);
        }
        __syncwarp();
    }
}

__global__ void gather_kernel(int n, int cap, const int32_t *__restrict__ idx, const double *__restrict__ x,
                              const double *__restrict__ y, const double *__restrict__ z,
                              const double *__restrict__ r, double *__restrict__ ps) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int i = idx[s];
        ps[s] = x[i];
        ps[cap + s] = y[i];
        ps[2 * (size_t)cap + s] = z[i];
        ps[3 * (size_t)cap + s] = r[i];
    }
}

__global__ void root_kernel(BhNodes nd, int n) {
    nd.start[0] = 0;
    nd.count[0] = n;
    nd.level[0] = 0;
    nd.first_child[0] = -1;
    nd.nchild[0] = 0;
}

// first index in [lo, hi) whose 3-bit digit at `shift` is >= o (digits are
// non-decreasing inside a node's run)
__device__ __forceinline__ int digit_lower_bound(const uint32_t *keys, int lo, int hi, int shift, uint32_t o) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (((keys[mid] >> shift) & 7u) < o)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Split points of the nodes [ls, le): eight lanes per node, lane o searching the first droplet
// of octant o over the whole node (the digits never decrease inside a node's run, so this
// equals a search that starts from octant o - 1's point) -- the eight searches run side by
// side instead of one after another, which matters for the few huge nodes of the top levels.
__global__ void level_count_kernel(BhNodes nd, const uint32_t *__restrict__ keys, int ls, int le, int leaf_size,
                                   int32_t *__restrict__ bounds, int M, int32_t *__restrict__ nchild_out) {
    const int lane = threadIdx.x & 31;
    const long long total = 8LL * (le - ls);
    const long long stride = (long long)gridDim.x * blockDim.x;
    // whole warps iterate together (the octant counts below are warp votes)
    for (long long base = (long long)blockIdx.x * blockDim.x + threadIdx.x - lane; base < total; base += stride) {
        const long long t = base + lane;
        const bool live = t < total;
        const int k = live ? ls + (int)(t >> 3) : ls, o = (int)(t & 7);
        int s0 = 0, c = 0, bo = 0;
        bool split = false;
        if (live) {
            s0 = nd.start[k];
            c = nd.count[k];
            split = c > leaf_size && nd.level[k] < BH_MAX_LEVEL;
            if (split) bo = o == 0 ? s0 : digit_lower_bound(keys, s0, s0 + c, 27 - 3 * nd.level[k], (uint32_t)o);
        }
        const int next = __shfl_down_sync(0xffffffffu, bo, 1);  // octant o + 1's point (lanes of one node)
        const int hi = o == 7 ? s0 + c : next;
        const unsigned nonempty = __ballot_sync(0xffffffffu, split && hi > bo);
        const int nch = __popc((nonempty >> (lane & ~7)) & 0xffu);
        if (live && split) {
            bounds[o * M + k] = bo;
            if (o == 7) bounds[8 * M + k] = s0 + c;
        }
        if (live && o == 0) {
            nd.nchild[k] = nch;
            nchild_out[k - ls] = nch;
        }
    }
}

__global__ void level_write_kernel(BhNodes nd, int ls, int le, const int32_t *__restrict__ bounds, int M,
                                   const int32_t *__restrict__ child_off, int next0) {
    for (int k = ls + blockIdx.x * blockDim.x + threadIdx.x; k < le; k += gridDim.x * blockDim.x) {
        const int nch = nd.nchild[k];
        if (nch == 0) {
            nd.first_child[k] = -1;
            continue;
        }
        int c = next0 + child_off[k - ls];
        nd.first_child[k] = c;
        const int lv = nd.level[k] + 1;
        for (int o = 0; o < 8; ++o) {
            const int a = bounds[o * M + k], b = bounds[(o + 1) * M + k];
            if (b > a) {
                nd.start[c] = a;
                nd.count[c] = b - a;
                nd.level[c] = lv;
                nd.first_child[c] = -1;
                nd.nchild[c] = 0;
                ++c;
            }
        }
    }
}

// Node k's R^3-weighted centre and second moment from its sums v (weight, first and
// second moments relative to (rx, ry, rz), the node's first droplet).
__device__ void r3_finish(BhNodes nd, int k, const double *v, double rx, double ry, double rz, int s0, int c, double ox,
                          double oy, double oz, double box, const uint32_t *__restrict__ keys) {
    {
        {
            const double w = v[0];
            float Q[6];
            if (w > 0.0) {
                const double mx = v[1] / w, my = v[2] / w, mz = v[3] / w;
                nd.cx[k] = rx + mx;
                nd.cy[k] = ry + my;
                nd.cz[k] = rz + mz;
                Q[0] = (float)(v[4] - w * mx * mx);
                Q[1] = (float)(v[5] - w * mx * my);
                Q[2] = (float)(v[6] - w * mx * mz);
                Q[3] = (float)(v[7] - w * my * my);
                Q[4] = (float)(v[8] - w * my * mz);
                Q[5] = (float)(v[9] - w * mz * mz);
            } else {  // geometric centre of the cell (octree_node.py:98-114)
                const int lv = nd.level[k];
                const uint32_t key = c > 0 ? keys[s0] : 0u;
                const uint32_t pre = lv > 0 ? key >> (30 - 3 * lv) << (30 - 3 * lv) : 0u;
                const double side = ldexp(box, -lv), cell = ldexp(box, -10);
                nd.cx[k] = ox + compact10(pre >> 2) * cell + side * 0.5;
                nd.cy[k] = oy + compact10(pre >> 1) * cell + side * 0.5;
                nd.cz[k] = oz + compact10(pre) * cell + side * 0.5;
                for (int q = 0; q < 6; ++q) Q[q] = 0.f;
            }
            nd.qr[2 * (size_t)k] = make_float4(Q[0], Q[1], Q[2], Q[3]);
            nd.qr[2 * (size_t)k + 1] = make_float4(Q[4], Q[5], (float)w, 0.f);
        }
    }
}

// Node moments bottom up, one level per launch (deepest first), one thread per node; every node
// keeps its FP64 sums in nd.mom ([22][M]: 10 R^3 sums, then 12 force sums), so each droplet is
// read once, by its leaf, and an inner node combines at most 8 children.
//
// R^3 sums relative to the node's first droplet r (as r3_finish expects): a leaf sums its droplets,
// w = r_j^3, S1 = sum w (x - r), S2 = sum w (x - r)(x - r)^T; an inner node adds its children's
// sums moved from the child's first droplet r_c to its own (its first child's): with delta = r_c - r,
//   W += W_c,  S1 += S1_c + W_c delta,  S2 += S2_c + S1_c delta^T + delta S1_c^T + W_c delta delta^T.
__global__ void node_r3_up_kernel(BhNodes nd, int a, int b, int M, const double *__restrict__ ps, int cap,
                                  const double *__restrict__ geom, const uint32_t *__restrict__ keys) {
    const double ox = geom[0], oy = geom[1], oz = geom[2], box = geom[3];
    for (int k = a + blockIdx.x * blockDim.x + threadIdx.x; k < b; k += gridDim.x * blockDim.x) {
        const int s0 = nd.start[k], c = nd.count[k], nch = nd.nchild[k];
        const double rx = c > 0 ? ps[s0] : 0.0, ry = c > 0 ? ps[cap + s0] : 0.0,
                     rz = c > 0 ? ps[2 * (size_t)cap + s0] : 0.0;
        double v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // w, w d (3), w d d^T (6)
        if (nch == 0) {
            for (int t = 0; t < c; ++t) {
                const double r = ps[3 * (size_t)cap + s0 + t];
                const double w = r * r * r;
                const double dx = ps[s0 + t] - rx, dy = ps[cap + s0 + t] - ry, dz = ps[2 * (size_t)cap + s0 + t] - rz;
                v[0] += w;
                v[1] += w * dx;
                v[2] += w * dy;
                v[3] += w * dz;
                v[4] += w * dx * dx;
                v[5] += w * dx * dy;
                v[6] += w * dx * dz;
                v[7] += w * dy * dy;
                v[8] += w * dy * dz;
                v[9] += w * dz * dz;
            }
        } else {
            const int f = nd.first_child[k];
            for (int q = 0; q < nch; ++q) {
                const int ch = f + q, cs0 = nd.start[ch];
                const double dx = ps[cs0] - rx, dy = ps[cap + cs0] - ry, dz = ps[2 * (size_t)cap + cs0] - rz;
                double u[10];
#pragma unroll
                for (int p = 0; p < 10; ++p) u[p] = nd.mom[(size_t)p * M + ch];
                v[0] += u[0];
                v[1] += u[1] + u[0] * dx;
                v[2] += u[2] + u[0] * dy;
                v[3] += u[3] + u[0] * dz;
                v[4] += u[4] + 2.0 * u[1] * dx + u[0] * dx * dx;
                v[5] += u[5] + u[1] * dy + dx * u[2] + u[0] * dx * dy;
                v[6] += u[6] + u[1] * dz + dx * u[3] + u[0] * dx * dz;
                v[7] += u[7] + 2.0 * u[2] * dy + u[0] * dy * dy;
                v[8] += u[8] + u[2] * dz + dy * u[3] + u[0] * dy * dz;
                v[9] += u[9] + 2.0 * u[3] * dz + u[0] * dz * dz;
            }
        }
#pragma unroll
        for (int p = 0; p < 10; ++p) nd.mom[(size_t)p * M + k] = v[p];
        r3_finish(nd, k, v, rx, ry, rz, s0, c, ox, oy, oz, box, keys);
    }
}

// Force sum F and dipole D = sum (x - c) F^T about the node's centre c: a leaf sums its droplets; an
// inner node adds its children's, moved to its centre: F += F_c, D += D_c + (c_c - c) F_c^T.
__global__ void node_force_up_kernel(BhNodes nd, int a, int b, int M, const double *__restrict__ ps,
                                     const double *__restrict__ fsort, int cap) {
    double *fm = nd.mom + (size_t)10 * M;
    for (int k = a + blockIdx.x * blockDim.x + threadIdx.x; k < b; k += gridDim.x * blockDim.x) {
        const int s0 = nd.start[k], c = nd.count[k], nch = nd.nchild[k];
        const double cx = nd.cx[k], cy = nd.cy[k], cz = nd.cz[k];
        double v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // F (3), D row-major (9)
        if (nch == 0) {
            for (int t = 0; t < c; ++t) {
                const int sj = s0 + t;
                const double F[3] = {fsort[sj], fsort[cap + sj], fsort[2 * (size_t)cap + sj]};
                const double d[3] = {ps[sj] - cx, ps[cap + sj] - cy, ps[2 * (size_t)cap + sj] - cz};
#pragma unroll
                for (int q = 0; q < 3; ++q) v[q] += F[q];
#pragma unroll
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int q = 0; q < 3; ++q) v[3 + 3 * p + q] += d[p] * F[q];
            }
        } else {
            const int f = nd.first_child[k];
            for (int q0 = 0; q0 < nch; ++q0) {
                const int ch = f + q0;
                const double d[3] = {nd.cx[ch] - cx, nd.cy[ch] - cy, nd.cz[ch] - cz};
                double u[12];
#pragma unroll
                for (int p = 0; p < 12; ++p) u[p] = fm[(size_t)p * M + ch];
#pragma unroll
                for (int q = 0; q < 3; ++q) v[q] += u[q];
#pragma unroll
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int q = 0; q < 3; ++q) v[3 + 3 * p + q] += u[3 + 3 * p + q] + d[p] * u[q];
            }
        }
#pragma unroll
        for (int p = 0; p < 12; ++p) fm[(size_t)p * M + k] = v[p];
        // v = (F, D row-major) -> the record: F, S (off-diagonal doubled), A = D^T - D
        nd.fd[3 * (size_t)k] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
        nd.fd[3 * (size_t)k + 1] =
            make_float4((float)v[7], (float)v[11], (float)(v[4] + v[6]), (float)(v[5] + v[9]));
        nd.fd[3 * (size_t)k + 2] =
            make_float4((float)(v[8] + v[10]), (float)(v[6] - v[4]), (float)(v[9] - v[5]), (float)(v[10] - v[8]));
    }
}

// ---------------------------------------------------------------------------
// walks
// ---------------------------------------------------------------------------
// Scaled units in FP32: lengths / ell (ell = 2^e with 2^(e-1) <= max r), forces
// * 2^-q (2^(q-1) <= max |F|).  Node aggregates are stored in these units:
// R^3 / ell^3, Q / ell^5, sum F 2^-q, D 2^-q / ell.
// (1/6) Q_ab d_a d_b d_c phi at x = D (see the file header); r7 = |x|^-7 etc.
__device__ __forceinline__ void quad_force(float x, float y, float z, const float4 qa, const float4 qb, float rinv,
                                           float rinv2, float &gx, float &gy, float &gz) {
    const float r7 = (rinv2 * rinv2) * (rinv2 * rinv), r9 = r7 * rinv2, r11 = r9 * rinv2;
    const float qxx = qa.x, qxy = qa.y, qxz = qa.z, qyy = qa.w, qyz = qb.x, qzz = qb.y;
    const float tr = qxx + qyy + qzz;
    const float Qx = fmaf(qxx, x, fmaf(qxy, y, qxz * z));
    const float Qy = fmaf(qxy, x, fmaf(qyy, y, qyz * z));
    const float Qz = fmaf(qxz, x, fmaf(qyz, y, qzz * z));
    const float xQx = fmaf(x, Qx, fmaf(y, Qy, z * Qz));
    // from |d|^-3: 15 [(tr x + 2 Q x) r^-7 - 7 (x.Qx) x r^-9]
    const float a1 = 15.f * r7, a2 = -105.f * xQx * r9;
    // from dz^2 |d|^-5 (times -3 below)
    const float b1 = 35.f * z * z * r9;
    const float b2 = -10.f * qzz * r7 + 140.f * z * Qz * r9 - 315.f * z * z * xQx * r11;
    const float tx = fmaf(2.f, Qx, tr * x), ty = fmaf(2.f, Qy, tr * y), tz = fmaf(2.f, Qz, tr * z);
    const float Bx = b1 * tx + b2 * x - 20.f * z * qxz * r7;
    const float By = b1 * ty + b2 * y - 20.f * z * qyz * r7;
    const float Bz = b1 * tz + b2 * z - 20.f * z * qzz * r7 - 20.f * Qz * r7 - 10.f * z * (tr * r7 - 7.f * xQx * r9);
    gx += (a1 * tx + a2 * x - 3.f * Bx) * (1.f / 6.f);
    gy += (a1 * ty + a2 * y - 3.f * By) * (1.f / 6.f);
    gz += (a1 * tz + a2 * z - 3.f * Bz) * (1.f / 6.f);
}

struct BhWalk {
    int n, cap, node_count;
    const double *ps;                  // sorted x, y, z, r (FP64, metres)
    const int32_t *idx;                // sorted -> caller order
    BhNodes nd;
    const double *geom;                // root cube origin and side
    const unsigned long long *scales;  // [0] max r, [1] max |F|
    const double *fsort;               // forces in sorted order (velocity walk)
    const float4 *loff;                // per sorted droplet: offset from its leaf's centre and radius, / ell
    const float4 *fs32;                // per sorted droplet: force * 2^-q (velocity walk)
    float theta2;
    int window_level;
    double L, halfL;
    unsigned long long *counters;  // [0] leaf pair terms, [1] accepted-node terms
    uint32_t *err;
    // periodic-image correction (velocity walk with CORR): FP32 grid view whose
    // slope corr.A is set per launch from corr_A (metres -> grid) and ell
    CorrF32 corr;
    double corr_A, corr_common, corr_self;
};

template <bool PER>
__device__ __forceinline__ double bh_mic(double d, double L, double halfL) {
    return PER ? mic64(d, L, halfL) : d;
}

// FORCE: F_i = m r_i^3 (sum_leaf r_j^3 P(d)/|d|^7 + sum_nodes R^3 P(D)/|D|^7), d = x_j - x_i, D = c - x_i
// else:  u_i = [F_i / (stokes r_i)] + eta (sum_leaf G(e) F_j + sum_nodes G(e) F_node + dipole), e = x_i - x_j
// CORR (velocity): + the periodic-image correction of every leaf pair and
// accepted node (FP32, summed apart) and, when stokes <= 0, the self term.
// Resident CTAs per SM asked of the register allocator (72 / 78-80 / 96 registers, none
// spilled): the force walk runs fastest at 6, the velocity walk at 7; the correction's extra
// live values fit at 5.
template <bool PER, bool FORCE, bool CORR = false>
__global__ void __launch_bounds__(BH_T, FORCE ? 6 : (CORR ? 5 : 7)) bh_walk_kernel(const BhWalk w, double coeff, double stokes,
                                                       double *__restrict__ ox, double *__restrict__ oy,
                                                       double *__restrict__ oz, double *__restrict__ fsort_out) {
    __shared__ int stack[BH_T / 32][BH_STACK];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int n = w.n, cap = w.cap;
    const double inv_ell = pow2_inv_of(w.scales[0]);
    const double fsc = FORCE ? 1.0 : pow2_inv_of(w.scales[1]);
    CorrF32 cf = w.corr;
    if (CORR) cf.A = (float)(w.corr_A / inv_ell);  // separations are in units of ell
    const float Ls = (float)(w.L * inv_ell), invLs = (float)(1.0 / (w.L * inv_ell));
    const float edge = (float)(w.L * inv_ell * (0.5 - 1e-6));  // leaf pairs: FP32 separations err by < 1e-6 L
    const double gox = w.geom[0], goy = w.geom[1], goz = w.geom[2];
    unsigned long long pairs = 0, nodes = 0;
    const int warps = gridDim.x * (BH_T / 32);
    for (int base = (blockIdx.x * (BH_T / 32) + wp) * 32; base < n; base += warps * 32) {
        const int si = base + lane;
        const bool valid = si < n;
        const int sl = valid ? si : base;  // padding lanes shadow a real droplet, their results are dropped
        const double xi = w.ps[sl], yi = w.ps[cap + sl], zi = w.ps[2 * (size_t)cap + sl],
                     ri = w.ps[3 * (size_t)cap + sl];
        // target in the nodes' FP32 frame (node separations: FP32, ~1e-6 relative for any accepted node)
        const float xs = (float)((xi - gox) * inv_ell), ys = (float)((yi - goy) * inv_ell),
                    zs = (float)((zi - goz) * inv_ell);
        const float ris = (float)(ri * inv_ell);
        float ax = 0.f, ay = 0.f, az = 0.f;
        float cx = 0.f, cy = 0.f, cz = 0.f;  // correction sums (CORR)
        int sp = 1;
        if (lane == 0) stack[wp][0] = 0;
        __syncwarp();
        int iters = 0;
        bool broken = false;
        while (sp > 0) {
            if (++iters > w.node_count + 1) {  // a tree is visited at most once per node
                broken = true;
                break;
            }
            const int node = stack[wp][--sp];
            __syncwarp();
            // every record of the node in one round of loads: the walk is bound by their latency
            const int4 mt = w.nd.meta[node];  // count, nchild, first child / droplet, level
            const float4 cs = w.nd.cs[node];
            const float4 rec = FORCE ? w.nd.qr[2 * (size_t)node + 1] : w.nd.fd[3 * (size_t)node];
            const float4 rq = FORCE ? w.nd.qr[2 * (size_t)node] : w.nd.fd[3 * (size_t)node + 1];
            const float4 rd = FORCE ? make_float4(0.f, 0.f, 0.f, 0.f) : w.nd.fd[3 * (size_t)node + 2];
            const int cnt = mt.x;
            if (mt.w & (FORCE ? BH_SKIP_FORCE : BH_SKIP_VEL)) continue;  // empty, or :861 / :1155
            float fnx = 0.f, fny = 0.f, fnz = 0.f, r3n = 0.f;
            if (FORCE) {
                r3n = rec.z;
            } else {
                fnx = rec.x;
                fny = rec.y;
                fnz = rec.z;
            }
            float dx = cs.x - xs, dy = cs.y - ys, dz = cs.z - zs;
            if (PER) {  // minimum image
                dx = fmaf(-Ls, rintf(dx * invLs), dx);
                dy = fmaf(-Ls, rintf(dy * invLs), dy);
                dz = fmaf(-Ls, rintf(dz * invLs), dz);
            }
            const float D2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float side = cs.w;
            bool accept = side * side < w.theta2 * D2 && D2 > 0.f;
            if (PER && w.window_level > 0 && (mt.w & BH_LEVEL_MASK) < w.window_level) {
                // cells larger than L / 2^window_level: the whole cell inside the target's
                // minimum-image window (else its droplets take different images)
                const float hw = (float)(w.halfL * inv_ell) - side;
                accept = accept && fabsf(dx) < hw && fabsf(dy) < hw && fabsf(dz) < hw;
            }
            accept = accept || !valid;
            if (__all_sync(0xffffffffu, accept)) {
                if (valid) {
                    ++nodes;
                    const float rinv = rsqrtf(D2), rinv2 = rinv * rinv;
                    if (FORCE) {  // D = c - x_i
                        const float b = r3n * (rinv2 * rinv2) * (rinv2 * rinv);
                        const float ang = fmaf(4.f * dz, dz, -fmaf(dx, dx, dy * dy));
                        ax = fmaf(b * ang, dx, ax);
                        ay = fmaf(b * ang, dy, ay);
                        az = fmaf(b * fmaf(2.f * dz, dz, -3.f * fmaf(dx, dx, dy * dy)), dz, az);
                        quad_force(dx, dy, dz, rq, rec, rinv, rinv2, ax, ay, az);
                    } else {  // e = x_i - c = -D
                        const float ex = -dx, ey = -dy, ez = -dz;
                        const float dot = fmaf(ex, fnx, fmaf(ey, fny, ez * fnz));
                        ax = fmaf(rinv, fmaf(ex, dot * rinv2, fnx), ax);
                        ay = fmaf(rinv, fmaf(ey, dot * rinv2, fny), ay);
                        az = fmaf(rinv, fmaf(ez, dot * rinv2, fnz), az);
                        // dipole: (D^T e - D e) = A e, e.D e = e.S e, tr D = tr S (records: see BhNodes.fd)
                        const float sxx = rec.w, syy = rq.x, szz = rq.y, sxy2 = rq.z, sxz2 = rq.w, syz2 = rd.x,
                                    a01 = rd.y, a02 = rd.z, a12 = rd.w;
                        const float Aex = a01 * ey + a02 * ez, Aey = a12 * ez - a01 * ex, Aez = -a02 * ex - a12 * ey;
                        const float tr = sxx + syy + szz;
                        const float q = ex * (sxx * ex + sxy2 * ey + sxz2 * ez) + ey * (syy * ey + syz2 * ez) +
                                        ez * (szz * ez);
                        const float rinv3 = rinv * rinv2, rinv5 = rinv3 * rinv2;
                        ax += rinv3 * (Aex - tr * ex) + 3.f * ex * q * rinv5;
                        ay += rinv3 * (Aey - tr * ey) + 3.f * ey * q * rinv5;
                        az += rinv3 * (Aez - tr * ez) + 3.f * ez * q * rinv5;
                        if (CORR) corr_pair32(cf, ex, ey, ez, fnx, fny, fnz, cx, cy, cz);
                    }
                }
                continue;
            }
            const int nch = mt.y;
            if (nch == 0) {  // leaf: exact pair terms (contact cut r^2 >= (r_i + r_j)^2)
                const int s0 = mt.z;
                if (valid) pairs += cnt;
                // d = x_j - x_i = (x_j - c_leaf) + MIC(c_leaf - x_i): the first part stored per droplet in
                // FP32, the second taken in FP64 once per leaf, so d carries ~1e-7 of |d|, not of |x|
                const float lx = (float)(bh_mic<PER>(w.nd.cx[node] - xi, w.L, w.halfL) * inv_ell),
                            ly = (float)(bh_mic<PER>(w.nd.cy[node] - yi, w.L, w.halfL) * inv_ell),
                            lz = (float)(bh_mic<PER>(w.nd.cz[node] - zi, w.L, w.halfL) * inv_ell);
                for (int k = 0; k < cnt; ++k) {
                    const int sj = s0 + k;
                    const float4 o = w.loff[sj];
                    float dx = o.x + lx, dy = o.y + ly, dz = o.z + lz;
                    // within 1e-6 L of the image boundary (or past it: a leaf reaching across L/2 in a
                    // shallow tree) the image and the separation come from the FP64 positions
                    if (PER && fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))) > edge) {
                        dx = (float)(bh_mic<PER>(w.ps[sj] - xi, w.L, w.halfL) * inv_ell);
                        dy = (float)(bh_mic<PER>(w.ps[cap + sj] - yi, w.L, w.halfL) * inv_ell);
                        dz = (float)(bh_mic<PER>(w.ps[2 * (size_t)cap + sj] - zi, w.L, w.halfL) * inv_ell);
                    }
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz)), rs = ris + o.w;
                    if (!valid || sj == si || r2 < rs * rs) continue;
                    const float rinv = rsqrtf(r2), rinv2 = rinv * rinv;
                    if (FORCE) {
                        const float rjs = o.w;
                        const float b = rjs * rjs * rjs * (rinv2 * rinv2) * (rinv2 * rinv);
                        const float ang = fmaf(4.f * dz, dz, -fmaf(dx, dx, dy * dy));
                        ax = fmaf(b * ang, dx, ax);
                        ay = fmaf(b * ang, dy, ay);
                        az = fmaf(b * fmaf(2.f * dz, dz, -3.f * fmaf(dx, dx, dy * dy)), dz, az);
                    } else {  // e = x_i - x_j = -d
                        const float4 fj = w.fs32[sj];
                        const float fx = fj.x, fy = fj.y, fz = fj.z;
                        const float ex = -dx, ey = -dy, ez = -dz;
                        const float dot = fmaf(ex, fx, fmaf(ey, fy, ez * fz));
                        ax = fmaf(rinv, fmaf(ex, dot * rinv2, fx), ax);
                        ay = fmaf(rinv, fmaf(ey, dot * rinv2, fy), ay);
                        az = fmaf(rinv, fmaf(ez, dot * rinv2, fz), az);
                        if (CORR) corr_pair32(cf, ex, ey, ez, fx, fy, fz, cx, cy, cz);
                    }
                }
                continue;
            }
            if (sp + nch > BH_STACK) {  // cannot happen for depth <= 10; kept bounded anyway
                broken = true;
                break;
            }
            if (lane < nch) stack[wp][sp + lane] = mt.z + lane;
            sp += nch;
            __syncwarp();
        }
        if (broken && lane == 0) raise_device_error(w.err, DEM_DEVERR_NODE_OVERFLOW);
        if (valid) {
            const int i = w.idx[si];
            double vx, vy, vz;
            if (FORCE) {  // F = m r_i^3 acc / ell
                const double f = coeff * ri * ri * ri * inv_ell;
                vx = f * ax;
                vy = f * ay;
                vz = f * az;
                fsort_out[si] = vx;
                fsort_out[cap + si] = vy;
                fsort_out[2 * (size_t)cap + si] = vz;
            } else {  // u = eta / (ell 2^-q) acc  (+ F / (stokes r))
                const double f = coeff * inv_ell / fsc;
                vx = f * ax;
                vy = f * ay;
                vz = f * az;
                if (stokes > 0.0) {
                    const double a = 1.0 / (stokes * ri);
                    vx += w.fsort[si] * a;
                    vy += w.fsort[cap + si] * a;
                    vz += w.fsort[2 * (size_t)cap + si] * a;
                }
                if (CORR) {  // sum of G F_scaled -> G F common
                    const double g = w.corr_common / fsc;
                    vx += g * cx;
                    vy += g * cy;
                    vz += g * cz;
                    if (!(stokes > 0.0)) {  // self term (Stokeslet walk only, flat_tree.py:1271-1276)
                        vx += w.corr_self * w.fsort[si];
                        vy += w.corr_self * w.fsort[cap + si];
                        vz += w.corr_self * w.fsort[2 * (size_t)cap + si];
                    }
                }
            }
            ox[i] = vx;
            oy[i] = vy;
            oz[i] = vz;
        }
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) {  // per-target counts, summed over the warp
        pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
        nodes += __shfl_xor_sync(0xffffffffu, nodes, o);
    }
    if (lane == 0) {
        atomicAdd(&w.counters[0], pairs);
        atomicAdd(&w.counters[1], nodes);
    }
}

// ---------------------------------------------------------------------------
// Two targets per lane: a warp walks 64 consecutive sorted targets (lane l holds
// targets base + l and base + 32 + l) and evaluates each accepted node and leaf
// pair for both at once in packed FP32x2 arithmetic.  The tree cut is the one
// the 64 targets need together (a node is opened when any target fails the
// acceptance test), and the per-node work -- pop, loads, tests, vote -- is
// shared by twice the targets.  Terms are the same expressions as
// bh_walk_kernel's, evaluated per lane of a float2.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 p_rsqrt(float2 v) { return make_float2(rsqrtf(v.x), rsqrtf(v.y)); }

template <bool PER>
__device__ __forceinline__ float2 p_mic(float2 d, float2 invL, float2 nL) {
    if (!PER) return d;
    const float2 u = p_add(p_fma(d, invL, dup2(RINT_MAGIC)), dup2(-RINT_MAGIC));  // rint(d / L)
    return p_fma(nL, u, d);
}

// quad_force for two targets: x, y, z = D = c - x_i per lane, r7 = |D|^-7, rinv2 = |D|^-2.  The same
// closed form, its terms collected by what they multiply (with the 1/6 folded in):
//   g += X x + P Qx + C Q e_z + c_z e_z,  P = 2 c_t,  X = c_t tr + c_x,  C = 10 z r^-7,
//   c_t = 2.5 r^-7 - 17.5 z^2 r^-9,
//   c_x = -17.5 (x.Qx) r^-9 + 5 Qzz r^-7 - 70 z (Qx)_z r^-9 + 157.5 z^2 (x.Qx) r^-11,
//   c_z = 10 (Qx)_z r^-7 + 5 z tr r^-7 - 35 z (x.Qx) r^-9
// (checked against quad_force's form to 1e-14 in FP64 on random separations and moments).
__device__ __forceinline__ void quad_force2(float2 x, float2 y, float2 z, const float4 qa, const float4 qb, float2 r7,
                                            float2 rinv2, float2 &gx, float2 &gy, float2 &gz) {
    const float2 r9 = p_mul(r7, rinv2);
    const float qxx = qa.x, qxy = qa.y, qxz = qa.z, qyy = qa.w, qyz = qb.x, qzz = qb.y;
    const float tr = qxx + qyy + qzz;
    const float2 Qx = p_fma(dup2(qxx), x, p_fma(dup2(qxy), y, p_mul(dup2(qxz), z)));
    const float2 Qy = p_fma(dup2(qxy), x, p_fma(dup2(qyy), y, p_mul(dup2(qyz), z)));
    const float2 Qz = p_fma(dup2(qxz), x, p_fma(dup2(qyz), y, p_mul(dup2(qzz), z)));
    const float2 xQx = p_fma(x, Qx, p_fma(y, Qy, p_mul(z, Qz)));
    const float2 zz = p_mul(z, z), u = p_mul(xQx, r9), zr7 = p_mul(z, r7);
    const float2 ct = p_fma(dup2(-17.5f), p_mul(zz, r9), p_mul(dup2(2.5f), r7));
    const float2 cx = p_fma(dup2(-17.5f), u,
                            p_fma(dup2(5.f * qzz), r7,
                                  p_fma(dup2(-70.f), p_mul(p_mul(z, Qz), r9),
                                        p_mul(dup2(157.5f), p_mul(p_mul(zz, u), rinv2)))));
    const float2 cz = p_fma(dup2(10.f), p_mul(Qz, r7), p_fma(dup2(5.f * tr), zr7, p_mul(dup2(-35.f), p_mul(z, u))));
    const float2 X = p_fma(ct, dup2(tr), cx), P = p_add(ct, ct), C = p_mul(dup2(10.f), zr7);
    gx = p_fma(X, x, p_fma(P, Qx, p_fma(C, dup2(qxz), gx)));
    gy = p_fma(X, y, p_fma(P, Qy, p_fma(C, dup2(qyz), gy)));
    gz = p_fma(X, z, p_fma(P, Qz, p_fma(C, dup2(qzz), p_add(gz, cz))));
}

// The pair force r_j^3 P(d) / |d|^7 (b = r_j^3 |d|^-7, per lane) added to (ax, ay, az).
__device__ __forceinline__ void mono_force2(float2 dx, float2 dy, float2 dz, float2 b, float2 &ax, float2 &ay,
                                            float2 &az) {
    const float2 zz = p_mul(dz, dz), xy2 = p_fma(dx, dx, p_mul(dy, dy));
    const float2 ang = p_fma(dup2(-1.f), xy2, p_mul(dup2(4.f), zz));   // 4 dz^2 - dx^2 - dy^2
    const float2 angz = p_fma(dup2(-3.f), xy2, p_mul(dup2(2.f), zz));  // 2 dz^2 - 3 dx^2 - 3 dy^2
    const float2 ba = p_mul(b, ang);
    ax = p_fma(ba, dx, ax);
    ay = p_fma(ba, dy, ay);
    az = p_fma(p_mul(b, angz), dz, az);
}

// The Stokeslet G(e) F / 8 pi eta without constants: (F + e (e.F) / |e|^2) / |e|, added to (ax, ay, az).
__device__ __forceinline__ void stokeslet2(float2 ex, float2 ey, float2 ez, float2 fx, float2 fy, float2 fz,
                                           float2 rinv, float2 rinv2, float2 &ax, float2 &ay, float2 &az) {
    const float2 dot = p_fma(ex, fx, p_fma(ey, fy, p_mul(ez, fz)));
    const float2 sc = p_mul(dot, rinv2);
    ax = p_fma(rinv, p_fma(ex, sc, fx), ax);
    ay = p_fma(rinv, p_fma(ey, sc, fy), ay);
    az = p_fma(rinv, p_fma(ez, sc, fz), az);
}

template <bool PER, bool FORCE>
__global__ void __launch_bounds__(BH_T, FORCE ? BH_WALK2_CTAS_FORCE : BH_WALK2_CTAS_VEL)
    bh_walk2_kernel(const BhWalk w, double coeff, double stokes, double *__restrict__ ox, double *__restrict__ oy,
                    double *__restrict__ oz, double *__restrict__ fsort_out) {
    __shared__ int stack[BH_T / 32][BH_STACK];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int n = w.n, cap = w.cap;
    const double inv_ell = pow2_inv_of(w.scales[0]);
    const double fsc = FORCE ? 1.0 : pow2_inv_of(w.scales[1]);
    const float Ls = (float)(w.L * inv_ell), invLs = (float)(1.0 / (w.L * inv_ell));
    const float2 nL2 = dup2(-Ls), invL2 = dup2(invLs);
    const float edge = (float)(w.L * inv_ell * (0.5 - 1e-6));  // leaf pairs: FP32 separations err by < 1e-6 L
    const double gox = w.geom[0], goy = w.geom[1], goz = w.geom[2];
    unsigned long long pairs = 0, nodes = 0;
    const int warps = gridDim.x * (BH_T / 32);
    for (int base = (blockIdx.x * (BH_T / 32) + wp) * 64; base < n; base += warps * 64) {
        const int si0 = base + lane, si1 = base + 32 + lane;
        const bool v0 = si0 < n, v1 = si1 < n;
        const int nv = (int)v0 + (int)v1;
        const int sl0 = v0 ? si0 : base, sl1 = v1 ? si1 : base;  // padding targets shadow a real droplet
        const double xi0 = w.ps[sl0], yi0 = w.ps[cap + sl0], zi0 = w.ps[2 * (size_t)cap + sl0],
                     ri0 = w.ps[3 * (size_t)cap + sl0];
        const double xi1 = w.ps[sl1], yi1 = w.ps[cap + sl1], zi1 = w.ps[2 * (size_t)cap + sl1],
                     ri1 = w.ps[3 * (size_t)cap + sl1];
        // targets in the nodes' FP32 frame
        const float2 xs = make_float2((float)((xi0 - gox) * inv_ell), (float)((xi1 - gox) * inv_ell));
        const float2 ys = make_float2((float)((yi0 - goy) * inv_ell), (float)((yi1 - goy) * inv_ell));
        const float2 zs = make_float2((float)((zi0 - goz) * inv_ell), (float)((zi1 - goz) * inv_ell));
        const float2 ris = make_float2((float)(ri0 * inv_ell), (float)(ri1 * inv_ell));
        const float2 nxs = make_float2(-xs.x, -xs.y), nys = make_float2(-ys.x, -ys.y), nzs = make_float2(-zs.x, -zs.y);
        float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax;
        int sp = 1;
        if (lane == 0) stack[wp][0] = 0;
        __syncwarp();
        int iters = 0;
        bool broken = false;
        while (sp > 0) {
            if (++iters > w.node_count + 1) {  // a tree is visited at most once per node
                broken = true;
                break;
            }
            const int node = stack[wp][--sp];
            __syncwarp();
            const int4 mt = w.nd.meta[node];  // count, nchild, first child / droplet, level | flags
            const float4 cs = w.nd.cs[node];
            const float4 rec = FORCE ? w.nd.qr[2 * (size_t)node + 1] : w.nd.fd[3 * (size_t)node];
            const float4 rq = FORCE ? w.nd.qr[2 * (size_t)node] : w.nd.fd[3 * (size_t)node + 1];
            const float4 rd = FORCE ? make_float4(0.f, 0.f, 0.f, 0.f) : w.nd.fd[3 * (size_t)node + 2];
            const int cnt = mt.x;
            if (mt.w & (FORCE ? BH_SKIP_FORCE : BH_SKIP_VEL)) continue;  // empty, or :861 / :1155
            // force walk: D = c - x_i; velocity walk: e = x_i - c (= -D, the minimum image is odd)
            float2 dx = FORCE ? p_add(dup2(cs.x), nxs) : p_add(xs, dup2(-cs.x));
            float2 dy = FORCE ? p_add(dup2(cs.y), nys) : p_add(ys, dup2(-cs.y));
            float2 dz = FORCE ? p_add(dup2(cs.z), nzs) : p_add(zs, dup2(-cs.z));
            dx = p_mic<PER>(dx, invL2, nL2);
            dy = p_mic<PER>(dy, invL2, nL2);
            dz = p_mic<PER>(dz, invL2, nL2);
            const float2 D2 = p_fma(dx, dx, p_fma(dy, dy, p_mul(dz, dz)));
            const float side = cs.w, s2 = side * side;
            bool acc0 = s2 < w.theta2 * D2.x && D2.x > 0.f, acc1 = s2 < w.theta2 * D2.y && D2.y > 0.f;
            if (PER && w.window_level > 0 && (mt.w & BH_LEVEL_MASK) < w.window_level) {
                const float hw = (float)(w.halfL * inv_ell) - side;
                acc0 = acc0 && fabsf(dx.x) < hw && fabsf(dy.x) < hw && fabsf(dz.x) < hw;
                acc1 = acc1 && fabsf(dx.y) < hw && fabsf(dy.y) < hw && fabsf(dz.y) < hw;
            }
            if (__all_sync(0xffffffffu, (acc0 || !v0) && (acc1 || !v1))) {
                if (nv) {
                    nodes += nv;
                    const float2 rinv = p_rsqrt(D2), rinv2 = p_mul(rinv, rinv);
                    if (FORCE) {
                        const float2 r7 = p_mul(p_mul(rinv2, rinv2), p_mul(rinv2, rinv));
                        mono_force2(dx, dy, dz, p_mul(dup2(rec.z), r7), ax, ay, az);
                        quad_force2(dx, dy, dz, rq, rec, r7, rinv2, ax, ay, az);
                    } else {
                        const float2 fnx = dup2(rec.x), fny = dup2(rec.y), fnz = dup2(rec.z);
                        stokeslet2(dx, dy, dz, fnx, fny, fnz, rinv, rinv2, ax, ay, az);
                        // dipole: D^T e, D e, e.D e, tr D (D_ab from the records, row a, column b)
                        // dipole: (D^T e - D e) = A e, e.D e = e.S e, tr D = tr S (records: see BhNodes.fd)
                        const float sxx = rec.w, syy = rq.x, szz = rq.y, sxy2 = rq.z, sxz2 = rq.w, syz2 = rd.x,
                                    a01 = rd.y, a02 = rd.z, a12 = rd.w;
                        const float2 ntr = dup2(-(sxx + syy + szz));
                        const float2 t1 = p_fma(dup2(sxx), dx, p_fma(dup2(sxy2), dy, p_mul(dup2(sxz2), dz)));
                        const float2 t2 = p_fma(dup2(syy), dy, p_mul(dup2(syz2), dz));
                        const float2 q = p_fma(dx, t1, p_fma(dy, t2, p_mul(p_mul(dup2(szz), dz), dz)));
                        const float2 rinv3 = p_mul(rinv, rinv2), rinv5 = p_mul(rinv3, rinv2);
                        const float2 q3 = p_mul(p_mul(dup2(3.f), q), rinv5);
                        // V = A e - tr e
                        const float2 Vx = p_fma(ntr, dx, p_fma(dup2(a01), dy, p_mul(dup2(a02), dz)));
                        const float2 Vy = p_fma(ntr, dy, p_fma(dup2(-a01), dx, p_mul(dup2(a12), dz)));
                        const float2 Vz = p_fma(ntr, dz, p_fma(dup2(-a02), dx, p_mul(dup2(-a12), dy)));
                        ax = p_fma(rinv3, Vx, p_fma(dx, q3, ax));
                        ay = p_fma(rinv3, Vy, p_fma(dy, q3, ay));
                        az = p_fma(rinv3, Vz, p_fma(dz, q3, az));
                    }
                }
                continue;
            }
            const int nch = mt.y;
            if (nch == 0) {  // leaf: exact pair terms (contact cut r^2 >= (r_i + r_j)^2)
                const int s0 = mt.z;
                pairs += (unsigned long long)cnt * nv;
                // d = x_j - x_i = (x_j - c_leaf) + MIC(c_leaf - x_i): the first part per droplet in FP32,
                // the second in FP64 once per leaf and target
                const double lcx = w.nd.cx[node], lcy = w.nd.cy[node], lcz = w.nd.cz[node];
                const float2 lx = make_float2((float)(bh_mic<PER>(lcx - xi0, w.L, w.halfL) * inv_ell),
                                              (float)(bh_mic<PER>(lcx - xi1, w.L, w.halfL) * inv_ell));
                const float2 ly = make_float2((float)(bh_mic<PER>(lcy - yi0, w.L, w.halfL) * inv_ell),
                                              (float)(bh_mic<PER>(lcy - yi1, w.L, w.halfL) * inv_ell));
                const float2 lz = make_float2((float)(bh_mic<PER>(lcz - zi0, w.L, w.halfL) * inv_ell),
                                              (float)(bh_mic<PER>(lcz - zi1, w.L, w.halfL) * inv_ell));
                // every droplet of the leaf lies within `reach` of its centre on each axis, so while
                // |l| + reach stays below the edge for both targets of every lane, no pair of the leaf
                // needs the image-boundary test: the warp takes the loop compiled without it
                const float reach = (FORCE ? rec : w.nd.qr[2 * (size_t)node + 1]).w;
                const bool near_edge =
                    PER && (fmaxf(fabsf(lx.x), fmaxf(fabsf(ly.x), fabsf(lz.x))) + reach >= 0.999f * edge ||
                            fmaxf(fabsf(lx.y), fmaxf(fabsf(ly.y), fabsf(lz.y))) + reach >= 0.999f * edge);
                auto leaf_pairs = [&](auto edge_tests) {
                    for (int k = 0; k < cnt; ++k) {
                        const int sj = s0 + k;
                        const float4 o = w.loff[sj];
                        float2 dx = p_add(dup2(o.x), lx), dy = p_add(dup2(o.y), ly), dz = p_add(dup2(o.z), lz);
                        // within 1e-6 L of the image boundary (or past it: a leaf reaching across L/2 in a
                        // shallow tree) the image and the separation come from the FP64 positions
                        if (PER && decltype(edge_tests)::value) {
                            if (fmaxf(fabsf(dx.x), fmaxf(fabsf(dy.x), fabsf(dz.x))) > edge) {
                                dx.x = (float)(bh_mic<PER>(w.ps[sj] - xi0, w.L, w.halfL) * inv_ell);
                                dy.x = (float)(bh_mic<PER>(w.ps[cap + sj] - yi0, w.L, w.halfL) * inv_ell);
                                dz.x = (float)(bh_mic<PER>(w.ps[2 * (size_t)cap + sj] - zi0, w.L, w.halfL) * inv_ell);
                            }
                            if (fmaxf(fabsf(dx.y), fmaxf(fabsf(dy.y), fabsf(dz.y))) > edge) {
                                dx.y = (float)(bh_mic<PER>(w.ps[sj] - xi1, w.L, w.halfL) * inv_ell);
                                dy.y = (float)(bh_mic<PER>(w.ps[cap + sj] - yi1, w.L, w.halfL) * inv_ell);
                                dz.y = (float)(bh_mic<PER>(w.ps[2 * (size_t)cap + sj] - zi1, w.L, w.halfL) * inv_ell);
                            }
                        }
                        const float2 r2 = p_fma(dx, dx, p_fma(dy, dy, p_mul(dz, dz)));
                        const float2 rs = p_add(ris, dup2(o.w)), rs2 = p_mul(rs, rs);
                        // excluded: padding target, the target itself, or closer than r_i + r_j
                        const bool e0 = !v0 || sj == si0 || r2.x < rs2.x, e1 = !v1 || sj == si1 || r2.y < rs2.y;
                        if (e0 && e1) continue;
                        const float2 rinv = p_rsqrt(make_float2(e0 ? 1.f : r2.x, e1 ? 1.f : r2.y));
                        const float2 rinv2 = p_mul(rinv, rinv);
                        const float2 keep = make_float2(e0 ? 0.f : 1.f, e1 ? 0.f : 1.f);
                        if (FORCE) {
                            const float rj3 = o.w * o.w * o.w;
                            const float2 r7 = p_mul(p_mul(rinv2, rinv2), p_mul(rinv2, rinv));
                            mono_force2(dx, dy, dz, p_mul(p_mul(dup2(rj3), keep), r7), ax, ay, az);
                        } else {  // G(e) with e = x_i - x_j = -d: G is even, so d serves
                            const float4 fj = w.fs32[sj];
                            stokeslet2(dx, dy, dz, dup2(fj.x), dup2(fj.y), dup2(fj.z), p_mul(rinv, keep), rinv2, ax, ay,
                                       az);
                        }
                    }
                };
                if (__any_sync(0xffffffffu, near_edge))
                    leaf_pairs(std::true_type{});
                else
                    leaf_pairs(std::false_type{});
                continue;
            }
            if (sp + nch > BH_STACK) {  // cannot happen for depth <= 10; kept bounded anyway
                broken = true;
                break;
            }
            if (lane < nch) stack[wp][sp + lane] = mt.z + lane;
            sp += nch;
            __syncwarp();
        }
        if (broken && lane == 0) raise_device_error(w.err, DEM_DEVERR_NODE_OVERFLOW);
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const bool valid = t ? v1 : v0;
            if (!valid) continue;
            const int si = t ? si1 : si0;
            const double ri = t ? ri1 : ri0;
            const float gx = t ? ax.y : ax.x, gy = t ? ay.y : ay.x, gz = t ? az.y : az.x;
            const int i = w.idx[si];
            double vx, vy, vz;
            if (FORCE) {  // F = m r_i^3 acc / ell
                const double f = coeff * ri * ri * ri * inv_ell;
                vx = f * gx;
                vy = f * gy;
                vz = f * gz;
                fsort_out[si] = vx;
                fsort_out[cap + si] = vy;
                fsort_out[2 * (size_t)cap + si] = vz;
            } else {  // u = eta / (ell 2^-q) acc  (+ F / (stokes r))
                const double f = coeff * inv_ell / fsc;
                vx = f * gx;
                vy = f * gy;
                vz = f * gz;
                if (stokes > 0.0) {
                    const double a = 1.0 / (stokes * ri);
                    vx += w.fsort[si] * a;
                    vy += w.fsort[cap + si] * a;
                    vz += w.fsort[2 * (size_t)cap + si] * a;
                }
            }
            ox[i] = vx;
            oy[i] = vy;
            oz[i] = vz;
        }
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) {  // per-target counts, summed over the warp
        pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
        nodes += __shfl_xor_sync(0xffffffffu, nodes, o);
    }
    if (lane == 0) {
        atomicAdd(&w.counters[0], pairs);
        atomicAdd(&w.counters[1], nodes);
    }
}

__global__ void forces_to_sorted_kernel(int n, int cap, const int32_t *__restrict__ idx, const double *__restrict__ fx,
                                        const double *__restrict__ fy, const double *__restrict__ fz,
                                        double *__restrict__ fsort) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int i = idx[s];
        fsort[s] = fx[i];
        fsort[cap + s] = fy[i];
        fsort[2 * (size_t)cap + s] = fz[i];
    }
}

// node aggregates in walk units: centre and side / ell, r3 / ell^3, q / ell^5 (what = 0);
// fs * 2^-q, dp * 2^-q / ell (what = 1)
// Per sorted droplet: offset from the centre of its leaf and radius, in units of ell.
__global__ void leaf_offsets_kernel(BhNodes nd, int nc, const double *__restrict__ ps, int cap,
                                    const unsigned long long *__restrict__ scales, float4 *__restrict__ loff) {
    const double inv_ell = pow2_inv_of(scales[0]);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
        if (nd.nchild[k] != 0) continue;
        const int s0 = nd.start[k], cnt = nd.count[k];
        const double cx = nd.cx[k], cy = nd.cy[k], cz = nd.cz[k];
        float reach = 0.f;
        for (int j = s0; j < s0 + cnt; ++j) {
            const float4 o = make_float4((float)((ps[j] - cx) * inv_ell), (float)((ps[cap + j] - cy) * inv_ell),
                                         (float)((ps[2 * (size_t)cap + j] - cz) * inv_ell),
                                         (float)(ps[3 * (size_t)cap + j] * inv_ell));
            loff[j] = o;
            reach = fmaxf(reach, fmaxf(fabsf(o.x), fmaxf(fabsf(o.y), fabsf(o.z))));
        }
        nd.qr[2 * (size_t)k + 1].w = reach;  // the leaf's largest |offset| on any axis (the walks' edge test)
    }
}

// Sorted forces scaled by 2^-q (the velocity walk's unit), FP32.
__global__ void scale_forces_kernel(int n, int cap, const double *__restrict__ fsort,
                                    const unsigned long long *__restrict__ scales, float4 *__restrict__ fs32) {
    const double fsc = pow2_inv_of(scales[1]);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        fs32[j] = make_float4((float)(fsort[j] * fsc), (float)(fsort[cap + j] * fsc),
                              (float)(fsort[2 * (size_t)cap + j] * fsc), 0.f);
}

__global__ void scale_nodes_kernel(BhNodes nd, int nc, const unsigned long long *scales, const double *geom,
                                   int what) {
    const double inv_ell = pow2_inv_of(scales[0]);
    const double fsc = pow2_inv_of(scales[1]);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
        if (what == 0) {
            const int nch = nd.nchild[k], cnt = nd.count[k];
            nd.cs[k] = make_float4((float)((nd.cx[k] - geom[0]) * inv_ell), (float)((nd.cy[k] - geom[1]) * inv_ell),
                                   (float)((nd.cz[k] - geom[2]) * inv_ell),
                                   (float)(ldexp(geom[3], -nd.level[k]) * inv_ell));
            const double s3 = inv_ell * inv_ell * inv_ell, s5 = s3 * inv_ell * inv_ell;
            float *qr = reinterpret_cast<float *>(nd.qr + 2 * (size_t)k);  // Q[0..5], R^3
            for (int q = 0; q < 6; ++q) qr[q] = (float)((double)qr[q] * s5);
            qr[6] = (float)((double)qr[6] * s3);
            // the skip threshold in the walk's units (ell is a power of two: the same decision as in metres)
            const bool skip = cnt == 0 || (double)qr[6] < 1e-30 * s3;
            nd.meta[k] = make_int4(cnt, nch, nch ? nd.first_child[k] : nd.start[k],
                                   nd.level[k] | (skip ? BH_SKIP_FORCE : 0) | (cnt == 0 ? BH_SKIP_VEL : 0));
        } else {
            float *fd = reinterpret_cast<float *>(nd.fd + 3 * (size_t)k);  // F[0..2], then S and A (linear in D)
            for (int q = 0; q < 3; ++q) fd[q] = (float)((double)fd[q] * fsc);
            for (int q = 3; q < 12; ++q) fd[q] = (float)((double)fd[q] * fsc * inv_ell);
            const double f0 = fd[0], f1 = fd[1], f2 = fd[2];  // force sum in units of 2^q newtons
            const double f2sum = __dadd_rn(__dadd_rn(__dmul_rn(f0, f0), __dmul_rn(f1, f1)), __dmul_rn(f2, f2));
            int4 mt = nd.meta[k];
            const bool skip = mt.x == 0 || f2sum < 1e-60 * (fsc * fsc);
            mt.w = (mt.w & ~BH_SKIP_VEL) | (skip ? BH_SKIP_VEL : 0);
            nd.meta[k] = mt;
        }
    }
}

}  // namespace

namespace dem {

static size_t ws_align(size_t b) { return (b + 255) & ~size_t(255); }

size_t morton_ws_bytes(int n) {
    const size_t tiles = (size_t)((n + RS_TILE - 1) / RS_TILE);
    return 4 * ws_align(4 * (size_t)n) + ws_align(4 * 2 * (256 * tiles + 1)) + ws_align(6 * 8) + ws_align(4 * 8);
}

MortonWs morton_ws_carve(void *base, int n) {
    const size_t tiles = (size_t)((n + RS_TILE - 1) / RS_TILE);
    char *p = static_cast<char *>(base);
    MortonWs w;
    w.keys[0] = reinterpret_cast<uint32_t *>(p);
    p += ws_align(4 * (size_t)n);
    w.keys[1] = reinterpret_cast<uint32_t *>(p);
    p += ws_align(4 * (size_t)n);
    w.idx[0] = reinterpret_cast<int32_t *>(p);
    p += ws_align(4 * (size_t)n);
    w.idx[1] = reinterpret_cast<int32_t *>(p);
    p += ws_align(4 * (size_t)n);
    w.hist = reinterpret_cast<int32_t *>(p);
    p += ws_align(4 * 2 * (256 * tiles + 1));
    w.bbox = reinterpret_cast<long long *>(p);
    p += ws_align(6 * 8);
    w.geom = reinterpret_cast<double *>(p);
    return w;
}

int morton_order(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, int periodic, double L,
                 const MortonWs &w, cudaStream_t s) {
    const int g = std::max(1, std::min((n + 255) / 256, 8 * ctx->sm_count));
    if (!periodic) {
        bbox_init_kernel<<<1, 32, 0, counted(s)>>>(w.bbox);
        bbox_kernel<<<g, 256, 0, counted(s)>>>(n, x, y, z, w.bbox);
    }
    geom_kernel<<<1, 32, 0, counted(s)>>>(periodic ? 1 : 0, L, w.bbox, w.geom);
    keys_kernel<<<g, 256, 0, counted(s)>>>(n, x, y, z, w.geom, w.keys[0], w.idx[0]);
    return radix_sort_pairs(ctx, n, w, s);
}

int radix_pass(dem_ctx *ctx, int n, const uint32_t *kin, const int32_t *vin, uint32_t *kout, int32_t *vout, int shift,
               int32_t *hist, cudaStream_t s) {
    const int tiles = (n + RS_TILE - 1) / RS_TILE;
    int32_t *off = hist + 256 * (size_t)tiles + 1;
    rs_hist_kernel<<<tiles, RS_T, 0, counted(s)>>>(n, kin, shift, tiles, hist);
    int rc = exclusive_scan<int32_t, int32_t>(ctx, hist, off, 256LL * tiles, s);
    if (rc) return rc;
    rs_scatter_kernel<<<tiles, RS_T, 0, counted(s)>>>(n, kin, vin, kout, vout, shift, tiles, off);
    return dem_check_launch(ctx, "radix pass");
}

int radix_sort_pairs(dem_ctx *ctx, int n, const MortonWs &w, cudaStream_t s) {
    const int tiles = (n + RS_TILE - 1) / RS_TILE;
    int32_t *hist = w.hist, *off = w.hist + 256 * (size_t)tiles + 1;
    int cur = 0, rc;
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 8 * pass;
        rs_hist_kernel<<<tiles, RS_T, 0, counted(s)>>>(n, w.keys[cur], shift, tiles, hist);
        if ((rc = exclusive_scan<int32_t, int32_t>(ctx, hist, off, 256LL * tiles, s))) return rc;
        rs_scatter_kernel<<<tiles, RS_T, 0, counted(s)>>>(n, w.keys[cur], w.idx[cur], w.keys[1 - cur],
                                                          w.idx[1 - cur], shift, tiles, off);
        cur = 1 - cur;
    }
    return dem_check_launch(ctx, "morton order");  // four passes: the result is back in buffer 0
}

}  // namespace dem

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <typename T>
static int bh_alloc(dem_ctx *ctx, T **p, size_t count, const char *what) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    return dem_check_cuda(ctx, cudaMalloc((void **)p, sizeof(T) * (count > 0 ? count : 1)), what);
}

static void bh_free_nodes(BhNodes &nd) {
    void *ptrs[] = {nd.start, nd.count, nd.first_child, nd.nchild, nd.level, nd.cx, nd.cy,
                    nd.cz,    nd.mom,   nd.cs,          nd.meta,   nd.qr,    nd.fd};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    nd = BhNodes{};
}

// (Re)allocates node arrays for m nodes, keeping the first `keep` nodes' topology.
static int bh_nodes_reserve(dem_bh *b, int m, int keep, cudaStream_t s) {
    if (m <= b->max_nodes) return DEM_OK;
    dem_ctx *ctx = b->ctx;
    BhNodes nn{};
    int rc;
    if ((rc = bh_alloc(ctx, &nn.start, m, "bh nodes")) || (rc = bh_alloc(ctx, &nn.count, m, "bh nodes")) ||
        (rc = bh_alloc(ctx, &nn.first_child, m, "bh nodes")) || (rc = bh_alloc(ctx, &nn.nchild, m, "bh nodes")) ||
        (rc = bh_alloc(ctx, &nn.level, m, "bh nodes")) || (rc = bh_alloc(ctx, &nn.cx, m, "bh nodes")) ||
        (rc = bh_alloc(ctx, &nn.cy, m, "bh nodes")) || (rc = bh_alloc(ctx, &nn.cz, m, "bh nodes")) ||
        (rc = bh_alloc(ctx, &nn.cs, m, "bh nodes")) || (rc = bh_alloc(ctx, &nn.meta, m, "bh nodes")) ||
        (rc = bh_alloc(ctx, &nn.mom, 22 * (size_t)m, "bh nodes")) ||
        (rc = bh_alloc(ctx, &nn.qr, 2 * (size_t)m, "bh nodes")) ||
        (rc = bh_alloc(ctx, &nn.fd, 3 * (size_t)m, "bh nodes"))) {
        bh_free_nodes(nn);
        return rc;
    }
    if (keep > 0) {
        int *src[] = {b->nd.start, b->nd.count, b->nd.first_child, b->nd.nchild, b->nd.level};
        int *dst[] = {nn.start, nn.count, nn.first_child, nn.nchild, nn.level};
        for (int q = 0; q < 5; ++q)
            if ((rc = dem_check_cuda(
                     ctx, cudaMemcpyAsync(dst[q], src[q], sizeof(int) * keep, cudaMemcpyDeviceToDevice, s), "bh nodes")))
                return rc;
        if ((rc = dem_check_cuda(ctx, cudaStreamSynchronize(s), "bh nodes"))) return rc;
    }
    if ((rc = bh_alloc(ctx, &b->bounds, 9 * (size_t)m, "bh nodes")) ||
        (rc = bh_alloc(ctx, &b->scan_in, (size_t)m + 1, "bh nodes")) ||
        (rc = bh_alloc(ctx, &b->coff, (size_t)m + 1, "bh nodes"))) {
        bh_free_nodes(nn);
        return rc;
    }
    bh_free_nodes(b->nd);
    b->nd = nn;
    b->max_nodes = m;
    return DEM_OK;
}

static void bh_free(dem_bh *b) {
    cudaSetDevice(b->ctx->device);
    bh_free_nodes(b->nd);
    void *ptrs[] = {b->keys[0], b->keys[1], b->idx[0],   b->idx[1], b->hist,    b->ps,  b->fsort, b->loff, b->fs32,
                    b->bounds,  b->bbox,    b->geom,     b->counters, b->scales, b->scan_in, b->coff};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    delete b;
}

static inline int grid_of(dem_ctx *ctx, long long work, int threads = 256) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 8LL * ctx->sm_count) g = 8LL * ctx->sm_count;
    return (int)g;
}

// One past the last node of level l.
static int level_end(const dem_bh *b, int l) { return l + 1 < b->nlevels ? b->level_off[l + 1] : b->node_count; }

extern "C" {

int dem_bh_create(dem_ctx *ctx, int capacity, dem_bh **out) {
    if (!ctx || !out || capacity < 1) return dem_set_error(ctx, DEM_E_INVALID, "bh: bad arguments");
    *out = nullptr;
    int rc = dem_check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (rc) return rc;
    dem_bh *b = new dem_bh();
    b->ctx = ctx;
    b->capacity = capacity;
    const size_t n = (size_t)capacity;
    const int tiles = (capacity + RS_TILE - 1) / RS_TILE;
    if ((rc = bh_alloc(ctx, &b->keys[0], n, "bh")) || (rc = bh_alloc(ctx, &b->keys[1], n, "bh")) ||
        (rc = bh_alloc(ctx, &b->idx[0], n, "bh")) || (rc = bh_alloc(ctx, &b->idx[1], n, "bh")) ||
        (rc = bh_alloc(ctx, &b->hist, 2 * (256 * (size_t)tiles + 1), "bh")) ||
        (rc = bh_alloc(ctx, &b->ps, 4 * n, "bh")) || (rc = bh_alloc(ctx, &b->fsort, 3 * n, "bh")) ||
        (rc = bh_alloc(ctx, &b->loff, n, "bh")) || (rc = bh_alloc(ctx, &b->fs32, n, "bh")) ||
        (rc = bh_alloc(ctx, &b->bbox, 6, "bh")) || (rc = bh_alloc(ctx, &b->geom, 4, "bh")) ||
        (rc = bh_alloc(ctx, &b->counters, 2, "bh")) || (rc = bh_alloc(ctx, &b->scales, 2, "bh")) ||
        (rc = bh_nodes_reserve(b, std::max(4096, capacity / 4), 0, nullptr))) {
        bh_free(b);
        return rc;
    }
    *out = b;
    return DEM_OK;
}

void dem_bh_destroy(dem_bh *b) {
    if (b) bh_free(b);
}

int dem_bh_build(dem_bh *b, int n, const double *x, const double *y, const double *z, const double *r, double L,
                 int periodic, int leaf_size, void *stream) {
    if (!b) return DEM_E_INVALID;
    dem_ctx *ctx = b->ctx;
    if (n < 0 || leaf_size < 1) return dem_set_error(ctx, DEM_E_INVALID, "bh: n >= 0 and leaf_size >= 1");
    if (n > b->capacity) return dem_set_error(ctx, DEM_E_CAPACITY, "bh: number of particles exceeds the capacity");
    if (periodic && !(L > 0)) return dem_set_error(ctx, DEM_E_INVALID, "periodic boundaries need L > 0");
    int rc = dem_check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    b->n = n;
    b->L = L;
    b->periodic = periodic ? 1 : 0;
    b->leaf_size = leaf_size;
    b->level_off.assign(1, 0);
    b->node_count = 0;
    b->nlevels = 0;
    if (n == 0) return DEM_OK;
    dem_prof_begin(ctx, "bh_build", s);
    if (!periodic) {
        bbox_init_kernel<<<1, 32, 0, counted(s)>>>(b->bbox);
        bbox_kernel<<<grid_of(ctx, n), 256, 0, counted(s)>>>(n, x, y, z, b->bbox);
    }
    geom_kernel<<<1, 32, 0, counted(s)>>>(b->periodic, L, b->bbox, b->geom);
    keys_kernel<<<grid_of(ctx, n), 256, 0, counted(s)>>>(n, x, y, z, b->geom, b->keys[0], b->idx[0]);
    // stable LSD radix sort of (key, index), 8-bit digits, 30-bit keys: 4 passes
    const int tiles = (n + RS_TILE - 1) / RS_TILE;
    int32_t *hist = b->hist, *off = b->hist + 256 * (size_t)tiles + 1;  // histogram, its exclusive scan
    int cur = 0;
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 8 * pass;
        rs_hist_kernel<<<tiles, RS_T, 0, counted(s)>>>(n, b->keys[cur], shift, tiles, hist);
        if ((rc = exclusive_scan<int32_t, int32_t>(ctx, hist, off, 256LL * tiles, s))) return rc;
        rs_scatter_kernel<<<tiles, RS_T, 0, counted(s)>>>(n, b->keys[cur], b->idx[cur], b->keys[1 - cur],
                                                          b->idx[1 - cur], shift, tiles, off);
        cur = 1 - cur;
    }
    // after an even number of passes the sorted arrays are back in buffer 0
    gather_kernel<<<grid_of(ctx, n), 256, 0, counted(s)>>>(n, b->capacity, b->idx[0], x, y, z, r, b->ps);
    if ((rc = dem_check_cuda(ctx, cudaMemsetAsync(b->scales, 0, 2 * sizeof(unsigned long long), s), "memset")))
        return rc;
    maxabs_kernel<<<grid_of(ctx, n), 256, 0, counted(s)>>>(n, r, nullptr, nullptr, b->scales);
    // octree level by level (the host learns each level's size: one synchronisation per level)
    root_kernel<<<1, 1, 0, counted(s)>>>(b->nd, n);
    int ls = 0, le = 1;
    while (le > ls) {
        const int width = le - ls;
        int total = 0;
        for (int attempt = 0; attempt < 2; ++attempt) {
            level_count_kernel<<<grid_of(ctx, 8LL * width), 256, 0, counted(s)>>>(b->nd, b->keys[0], ls, le,
                                                                                 leaf_size, b->bounds, b->max_nodes,
                                                                                 b->scan_in);
            if ((rc = exclusive_scan<int32_t, int32_t>(ctx, b->scan_in, b->coff, width, s))) return rc;
            if ((rc = dem_check_cuda(
                     ctx, cudaMemcpyAsync(&total, b->coff + width, sizeof(int), cudaMemcpyDeviceToHost, s),
                     "bh level size")) ||
                (rc = dem_check_cuda(ctx, cudaStreamSynchronize(s), "bh level size")))
                return rc;
            if ((long long)le + total > 0x7fffffffLL) return dem_set_error(ctx, DEM_E_CAPACITY, "bh: too many nodes");
            if (le + total <= b->max_nodes) break;
            // grow the node arrays (the first le nodes are kept) and count this level again
            if ((rc = bh_nodes_reserve(b, std::max(le + total, 2 * b->max_nodes), le, s))) return rc;
        }
        if (total == 0) break;
        level_write_kernel<<<grid_of(ctx, width), 256, 0, counted(s)>>>(b->nd, ls, le, b->bounds, b->max_nodes,
                                                                       b->coff, le);
        b->level_off.push_back(le);
        ls = le;
        le += total;
    }
    b->node_count = le;
    b->nlevels = (int)b->level_off.size();
    // node R^3 and centres, bottom up (the deepest level first)
    for (int l = b->nlevels - 1; l >= 0; --l) {
        const int a = b->level_off[l], e = level_end(b, l);
        node_r3_up_kernel<<<grid_of(ctx, e - a), 256, 0, counted(s)>>>(b->nd, a, e, b->max_nodes, b->ps,
                                                                       b->capacity, b->geom, b->keys[0]);
    }
    scale_nodes_kernel<<<grid_of(ctx, le), 256, 0, counted(s)>>>(b->nd, le, b->scales, b->geom, 0);
    leaf_offsets_kernel<<<grid_of(ctx, le), 256, 0, counted(s)>>>(b->nd, le, b->ps, b->capacity, b->scales,
                                                                   b->loff);
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "bh build");
}

static BhWalk walk_args(dem_bh *b, float theta) {
    BhWalk w;
    w.n = b->n;
    w.cap = b->capacity;
    w.node_count = b->node_count;
    w.ps = b->ps;
    w.idx = b->idx[0];
    w.nd = b->nd;
    w.geom = b->geom;
    w.scales = b->scales;
    w.fsort = b->fsort;
    w.loff = b->loff;
    w.fs32 = b->fs32;
    w.theta2 = theta * theta;
    w.window_level = b->window_level;
    w.L = b->L;
    w.halfL = 0.5 * b->L;
    w.counters = b->counters;
    w.err = b->ctx->d_err;
    w.corr = CorrF32{};
    w.corr_A = w.corr_common = w.corr_self = 0.0;
    if (b->corr) {
        w.corr = corr_f32(b->corr, 1.0);
        w.corr_A = b->corr->cL * b->corr->ginv;
        w.corr_common = b->corr->common;
        w.corr_self = b->corr->g_self;
    }
    return w;
}

static int walk_grid(dem_bh *b) { return std::max(1, (b->n + BH_T - 1) / BH_T); }
// bh_walk2_kernel: 64 targets per warp
static int walk2_grid(dem_bh *b) { return std::max(1, (b->n + 2 * BH_T - 1) / (2 * BH_T)); }

int dem_bh_forces(dem_bh *b, double m_const, double theta, double *fx, double *fy, double *fz, void *stream) {
    if (!b || !(theta >= 0)) return DEM_E_INVALID;
    dem_ctx *ctx = b->ctx;
    cudaStream_t s = (cudaStream_t)stream;
    if (b->n == 0) return DEM_OK;
    int rc = dem_check_cuda(ctx, cudaMemsetAsync(b->counters, 0, 2 * sizeof(unsigned long long), s), "memset");
    if (rc) return rc;
    const BhWalk w = walk_args(b, (float)theta);
    dem_prof_begin(ctx, "bh_force_walk", s);
    if (b->periodic)
        bh_walk2_kernel<true, true><<<walk2_grid(b), BH_T, 0, counted(s)>>>(w, m_const, 0.0, fx, fy, fz, b->fsort);
    else
        bh_walk2_kernel<false, true><<<walk2_grid(b), BH_T, 0, counted(s)>>>(w, m_const, 0.0, fx, fy, fz, b->fsort);
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "bh force walk");
}

int dem_bh_velocity(dem_bh *b, const double *fx, const double *fy, const double *fz, double eta_const, double theta,
                    double stokes_factor, double *vx, double *vy, double *vz, void *stream) {
    if (!b || !(theta >= 0)) return DEM_E_INVALID;
    dem_ctx *ctx = b->ctx;
    cudaStream_t s = (cudaStream_t)stream;
    if (b->n == 0) return DEM_OK;
    const int n = b->n, le = b->node_count;
    int rc;
    if (fx)  // forces given in caller order (else: those of the last dem_bh_forces, already sorted)
        forces_to_sorted_kernel<<<grid_of(ctx, n), 256, 0, counted(s)>>>(n, b->capacity, b->idx[0], fx, fy, fz,
                                                                         b->fsort);
    const double *fs = b->fsort;
    if ((rc = dem_check_cuda(ctx, cudaMemsetAsync(b->scales + 1, 0, sizeof(unsigned long long), s), "memset")))
        return rc;
    maxabs_kernel<<<grid_of(ctx, n), 256, 0, counted(s)>>>(n, fs, fs + b->capacity, fs + 2 * (size_t)b->capacity,
                                                           b->scales + 1);
    for (int l = b->nlevels - 1; l >= 0; --l) {  // force sums and dipoles, bottom up
        const int a = b->level_off[l], e = level_end(b, l);
        node_force_up_kernel<<<grid_of(ctx, e - a), 256, 0, counted(s)>>>(b->nd, a, e, b->max_nodes, b->ps,
                                                                          b->fsort, b->capacity);
    }
    scale_nodes_kernel<<<grid_of(ctx, le), 256, 0, counted(s)>>>(b->nd, le, b->scales, b->geom, 1);
    scale_forces_kernel<<<grid_of(ctx, n), 256, 0, counted(s)>>>(n, b->capacity, b->fsort, b->scales, b->fs32);
    if ((rc = dem_check_cuda(ctx, cudaMemsetAsync(b->counters, 0, 2 * sizeof(unsigned long long), s), "memset")))
        return rc;
    const BhWalk w = walk_args(b, (float)theta);
    dem_prof_begin(ctx, "bh_velocity_walk", s);
    if (b->corr) {
        if (b->periodic)
            bh_walk_kernel<true, false, true><<<walk_grid(b), BH_T, 0, counted(s)>>>(w, eta_const, stokes_factor, vx,
                                                                                     vy, vz, nullptr);
        else
            bh_walk_kernel<false, false, true><<<walk_grid(b), BH_T, 0, counted(s)>>>(w, eta_const, stokes_factor, vx,
                                                                                      vy, vz, nullptr);
    } else if (b->periodic) {
        bh_walk2_kernel<true, false><<<walk2_grid(b), BH_T, 0, counted(s)>>>(w, eta_const, stokes_factor, vx, vy, vz,
                                                                             nullptr);
    } else {
        bh_walk2_kernel<false, false><<<walk2_grid(b), BH_T, 0, counted(s)>>>(w, eta_const, stokes_factor, vx, vy,
                                                                              vz, nullptr);
    }
    dem_prof_end(ctx, s);
    return dem_check_launch(ctx, "bh velocity walk");
}

int dem_bh_set_correction(dem_bh *b, const dem_corr *corr) {
    if (!b) return DEM_E_INVALID;
    if (corr && corr->ctx && corr->ctx->device != b->ctx->device)
        return dem_set_error(b->ctx, DEM_E_INVALID, "correction grid lives on another device");
    b->corr = corr;
    return DEM_OK;
}

int dem_bh_set_window(dem_bh *b, int window_level) {
    if (!b || window_level < 0) return DEM_E_INVALID;
    b->window_level = window_level;
    return DEM_OK;
}

int dem_bh_stats(dem_bh *b, int64_t *out) {
    if (!b || !out) return DEM_E_INVALID;
    unsigned long long c[2] = {0, 0};
    int rc = dem_check_cuda(b->ctx, cudaMemcpy(c, b->counters, sizeof(c), cudaMemcpyDeviceToHost), "bh stats");
    if (rc) return rc;
    out[0] = b->node_count;
    out[1] = b->nlevels;
    out[2] = b->n;
    out[3] = b->max_nodes;
    out[4] = (int64_t)c[0];
    out[5] = (int64_t)c[1];
    out[6] = b->leaf_size;
    out[7] = b->capacity;
    return DEM_OK;
}

}  // extern "C"
