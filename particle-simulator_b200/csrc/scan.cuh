// scan.cuh -- exclusive prefix sums on the device (three-phase: block totals,
// scan of the totals by one CTA, rescan with offsets).  Deterministic.
#pragma once

#include "common.cuh"

namespace dem {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;  // elements per CTA
constexpr int SCAN_MAX_BLOCKS = 1024 * 8;             // => up to 33.5M elements

// out[k] = sum(in[0..k)) for k in [0, n]; out has n + 1 slots (out[n] = total).
// The input may be a transform of `in`: op(in[k]) (e.g. flag != 0).
template <typename TIn, typename TOut>
int exclusive_scan(dem_ctx *ctx, const TIn *in, TOut *out, int64_t n, cudaStream_t s);

// Same scan with a caller-provided workspace of SCAN_MAX_BLOCKS + 1 TOut
// values (no context, no allocation).  Returns a cudaError_t value.
template <typename TIn, typename TOut>
cudaError_t exclusive_scan_into(const TIn *in, TOut *out, int64_t n, TOut *sums, cudaStream_t s);

}  // namespace dem
