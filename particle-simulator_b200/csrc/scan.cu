// scan.cu -- see scan.cuh.
#include "scan.cuh"

namespace dem {

template <typename T>
__device__ __forceinline__ T warp_inclusive(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan of one value per thread across the CTA; returns the CTA total.
template <typename T>
__device__ __forceinline__ T block_exclusive(T v, T *warp_sums, T &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    T inc = warp_inclusive(v);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nwarps ? warp_sums[lane] : T(0);
        T wi = warp_inclusive(w);
        if (lane < nwarps) warp_sums[lane] = wi - w;
        if (lane == nwarps - 1) warp_sums[32] = wi;
    }
    __syncthreads();
    total = warp_sums[32];
    T r = warp_sums[warp] + inc - v;
    __syncthreads();
    return r;
}

template <typename TIn, typename TOut>
__global__ void __launch_bounds__(SCAN_THREADS) scan_block_totals(const TIn *__restrict__ in, int64_t n,
                                                                 TOut *__restrict__ sums) {
    __shared__ TOut ws[33];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    TOut acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < n) acc += (TOut)in[base + k];
    TOut total;
    block_exclusive<TOut>(acc, ws, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename TOut>
__global__ void __launch_bounds__(1024) scan_totals(TOut *__restrict__ sums, int nb) {
    __shared__ TOut ws[33];
    constexpr int ITEMS = SCAN_MAX_BLOCKS / 1024;
    const int base = threadIdx.x * ITEMS;
    TOut v[ITEMS];
    TOut acc = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        v[k] = base + k < nb ? sums[base + k] : TOut(0);
        acc += v[k];
    }
    TOut total;
    TOut off = block_exclusive<TOut>(acc, ws, total);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        if (base + k < nb) sums[base + k] = off;
        off += v[k];
    }
    if (threadIdx.x == 0) sums[SCAN_MAX_BLOCKS] = total;
}

template <typename TIn, typename TOut>
__global__ void __launch_bounds__(SCAN_THREADS) scan_apply(const TIn *__restrict__ in, int64_t n,
                                                           const TOut *__restrict__ sums, TOut *__restrict__ out) {
    __shared__ TOut ws[33];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    TOut v[SCAN_ITEMS];
    TOut acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = base + k < n ? (TOut)in[base + k] : TOut(0);
        acc += v[k];
    }
    TOut total;
    TOut off = block_exclusive<TOut>(acc, ws, total) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = off;
        off += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = sums[SCAN_MAX_BLOCKS];
}

template <typename TIn, typename TOut>
int exclusive_scan(dem_ctx *ctx, const TIn *in, TOut *out, int64_t n, cudaStream_t s) {
    const int64_t nb64 = n > 0 ? (n + SCAN_TILE - 1) / SCAN_TILE : 1;
    if (nb64 > SCAN_MAX_BLOCKS) return dem_set_error(ctx, DEM_E_CAPACITY, "scan: too many elements");
    const int nb = (int)nb64;
    const size_t need = sizeof(int64_t) * (SCAN_MAX_BLOCKS + 1);
    if (ctx->scan_tmp_bytes < need) {
        if (ctx->scan_tmp) cudaFree(ctx->scan_tmp);
        ctx->scan_tmp = nullptr;
        ctx->scan_tmp_bytes = 0;
        int rc = dem_check_cuda(ctx, cudaMalloc(&ctx->scan_tmp, need), "scan workspace");
        if (rc) return rc;
        ctx->scan_tmp_bytes = need;
    }
    TOut *sums = reinterpret_cast<TOut *>(ctx->scan_tmp);
    scan_block_totals<TIn, TOut><<<nb, SCAN_THREADS, 0, counted(s)>>>(in, n, sums);
    scan_totals<TOut><<<1, 1024, 0, counted(s)>>>(sums, nb);
    scan_apply<TIn, TOut><<<nb, SCAN_THREADS, 0, counted(s)>>>(in, n, sums, out);
    return dem_check_launch(ctx, "exclusive_scan");
}

template <typename TIn, typename TOut>
cudaError_t exclusive_scan_into(const TIn *in, TOut *out, int64_t n, TOut *sums, cudaStream_t s) {
    const int64_t nb64 = n > 0 ? (n + SCAN_TILE - 1) / SCAN_TILE : 1;
    if (nb64 > SCAN_MAX_BLOCKS) return cudaErrorInvalidValue;
    const int nb = (int)nb64;
    scan_block_totals<TIn, TOut><<<nb, SCAN_THREADS, 0, counted(s)>>>(in, n, sums);
    scan_totals<TOut><<<1, 1024, 0, counted(s)>>>(sums, nb);
    scan_apply<TIn, TOut><<<nb, SCAN_THREADS, 0, counted(s)>>>(in, n, sums, out);
    return cudaGetLastError();
}

template cudaError_t exclusive_scan_into<int32_t, int32_t>(const int32_t *, int32_t *, int64_t, int32_t *,
                                                            cudaStream_t);
template cudaError_t exclusive_scan_into<int32_t, int64_t>(const int32_t *, int64_t *, int64_t, int64_t *,
                                                            cudaStream_t);

template int exclusive_scan<int32_t, int32_t>(dem_ctx *, const int32_t *, int32_t *, int64_t, cudaStream_t);
template int exclusive_scan<int32_t, int64_t>(dem_ctx *, const int32_t *, int64_t *, int64_t, cudaStream_t);
template int exclusive_scan<uint8_t, int32_t>(dem_ctx *, const uint8_t *, int32_t *, int64_t, cudaStream_t);

}  // namespace dem
