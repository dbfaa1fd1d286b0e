// sym.cuh -- box tables of the symmetric mixed-precision passes.
//
// A pass runs over one or more independent periodic boxes ("boxes" of an
// ensemble).  Droplets of box b are [off[b], off[b+1]) of the caller's arrays;
// the packed layout pads every box to whole blocks of B = 128 * IPT droplets,
// so box b occupies [poff[b], poff[b+1]) of it; the block pairs (I <= J) of all
// boxes are numbered consecutively, box b owning items [ioff[b], ioff[b+1]).
#pragma once

#include "mixed_common.cuh"

namespace dem {

constexpr int SYM_T = 128;  // threads per CTA of the pair kernel (4 warps); TJ == SYM_T

struct SymBoxes {
    int nbox;
    int n_total, npad_total, items_total;
    // nbox == 1: the single box is described by these values
    int n1, npad1;
    double L1;
    const unsigned long long *scales1;  // [2]
    // nbox > 1: device arrays
    const int *off, *poff, *ioff;       // [nbox + 1]
    const double *L;                    // [nbox]
    const unsigned long long *scales;   // [nbox][2]: max r, max |F| (bit patterns)
};

// largest b in [0, nbox) with a[b] <= q (a non-decreasing, a[0] <= q)
__host__ __device__ __forceinline__ int box_index(const int *a, int nbox, int q) {
    int lo = 0, hi = nbox - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a[mid] <= q)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Bytes of the workspace of a pass: packed layout (64 bytes per padded
// droplet) followed by the i- and j-side partial sums of every block pair.
size_t sym_workspace_bytes(long long npad_total, long long items_total, int B);
// Bytes that follow it for the passes on droplets in Morton order (the order,
// per-block bounds and occupancy bitmaps).
size_t sym_sorted_extra_bytes(long long n_total, long long npad_total, long long items_total, int B);

// One symmetric pass over the boxes of `t`.  The scale slots (max r; max |F|
// for convection) must already hold this call's values.  `m` carries the FP64
// inputs (x, y, z, r; fx, fy, fz for convection) and the error word.
// ctas = 0: one CTA per block pair; otherwise a persistent grid of that many.
template <bool FORCE>
int run_sym_boxes(dem_ctx *ctx, const SymBoxes &t, int ipt, int ctas, bool per, const MixedArgs &m, double *work,
                  double coeff, double *ox, double *oy, double *oz, cudaStream_t s);

// Per-box maximum |v| over up to three arrays into scales[2 b + slot].
int launch_maxabs_boxes(dem_ctx *ctx, const SymBoxes &t, const double *a, const double *b, const double *c,
                        unsigned long long *scales, int slot, cudaStream_t s);

// Resident CTAs per SM of the pair kernel (for persistent grids).
int sym_resident_ctas(int ipt, bool per, bool force);

}  // namespace dem
