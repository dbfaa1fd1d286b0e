// morton.cuh -- droplets in Morton (Z-order) of 30-bit keys, on the device.
//
// Keys interleave 10 bits per axis of the cell of each droplet in the root
// cube ([0, L)^3 in a periodic box, else the droplets' bounding cube); a stable
// LSD radix sort (four 8-bit passes) orders (key, index).  Used by the
// Barnes-Hut build (bh.cu) and by the symmetric direct passes, whose blocks of
// consecutive droplets in this order are compact in space.
#pragma once

#include "common.cuh"

namespace dem {

struct MortonWs {
    uint32_t *keys[2];
    int32_t *idx[2];
    int32_t *hist;     // 2 * (256 * tiles + 1)
    long long *bbox;   // 6
    double *geom;      // 4: root cube origin and side
};

// Bytes of the workspace for n droplets (256-byte aligned regions).
size_t morton_ws_bytes(int n);
// Carves the workspace out of `base` (256-byte aligned).
MortonWs morton_ws_carve(void *base, int n);
// idx[0][k] = the droplet with the k-th smallest key (ties in index order);
// keys[0] holds the sorted keys.  n >= 1.
int morton_order(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, int periodic, double L,
                 const MortonWs &w, cudaStream_t s);
// Stable sort of (keys[0][k], idx[0][k]) by key, k < n: four 8-bit passes; the
// result is back in keys[0] / idx[0].
int radix_sort_pairs(dem_ctx *ctx, int n, const MortonWs &w, cudaStream_t s);
// One stable pass on the 8-bit digit (key >> shift) & 255: (kin, vin) -> (kout, vout).
int radix_pass(dem_ctx *ctx, int n, const uint32_t *kin, const int32_t *vin, uint32_t *kout, int32_t *vout, int shift,
               int32_t *hist, cudaStream_t s);

}  // namespace dem
