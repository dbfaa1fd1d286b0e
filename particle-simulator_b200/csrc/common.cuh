// common.cuh -- shared device helpers and the context layout of libdem_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "dem_b200.h"

#define DEM_HD __host__ __device__ __forceinline__

// ---------------------------------------------------------------------------
// Context.  The library owns its workspace; the caller owns inputs/outputs.
// ---------------------------------------------------------------------------
struct dem_mixed_tuning {
    int i_per_thread = 4;
    int threads = 128;
    int j_splits = 0;  // 0: choose from the SM count
    double near_force = 5.0;
    double near_oseen = 3.0;
    int schedule = 0;  // DEM_SCHED_AUTO / DEM_SCHED_SPLIT / DEM_SCHED_SYMMETRIC
};

struct dem_prof_rec {
    const char *name;
    cudaEvent_t start, stop;
};

struct dem_ctx {
    int device = 0;
    // opt-in kernel timing: CUDA events around the main kernels, on their stream
    bool prof_enabled = false;
    std::vector<dem_prof_rec> prof;
    std::vector<cudaEvent_t> prof_pool;
    int capacity = 0;
    int sm_count = 148;
    std::string last_error;
    dem_mixed_tuning tuning;

    // device error word (DEM_DEVERR_* bits)
    uint32_t *d_err = nullptr;

    // workspace, sized by capacity (see dem_ctx_reserve)
    float4 *pack_a = nullptr;   // mixed: (x, y, z, r^3) or (x, y, z, -) scaled, per particle
    float4 *pack_b = nullptr;   // mixed: (Fx, Fy, Fz, k r) scaled, per particle
    double *partial = nullptr;  // mixed: [splits][3][capacity] chunk partial sums
    double *sym_partial = nullptr;  // mixed, symmetric schedule: per block-pair partial sums
    size_t sym_partial_bytes = 0;
    // The Morton permutation a symmetric pass left in its workspace, and the layout it was
    // made for.  A caller that runs the convection pass on the positions of the force pass it
    // just ran (dem_direct_forces_and_convection, dem_batch_step) sets sym_reuse_order for
    // that pass, which then skips the sort when the layout matches.
    struct {
        const void *work = nullptr;
        int n_total = -1, npad_total = -1, nbox = 0, ipt = 0, per = -1;
    } sym_order;
    bool sym_reuse_order = false;
    int partial_splits = 0;
    double *dscratch = nullptr;     // 8 doubles: reductions (max radius, ...)
    int32_t *cell_hash = nullptr;   // hash bucket per particle
    int32_t *cell_xyz = nullptr;    // cell coordinates per particle, [3][capacity] (the count pass)
    int32_t *bucket_count = nullptr;  // table
    int32_t *bucket_start = nullptr;  // table (exclusive scan)
    int32_t *bucket_cursor = nullptr; // table
    int32_t *sorted_idx = nullptr;    // particles grouped by bucket
    double2 *hash_pos = nullptr;      // (x, y), (z, r) of the particles in bucket order (2 per particle)
    float4 *hash_pos32 = nullptr;     // (x, y, z, r) rounded to FP32, bucket order (the far test)
    int32_t *pair_count = nullptr;    // per particle (capacity + 1)
    int64_t *pair_offset = nullptr;   // per particle (capacity + 1), exclusive scan
    int64_t table_capacity = 0;
    int32_t *flags = nullptr;       // merge: 1 = consumed
    int32_t *keep_off = nullptr;    // merge: exclusive scan of survivors (capacity + 1)
    double *merged_buf = nullptr;   // merge: 4 doubles per merged droplet
    int32_t *merged_cnt = nullptr;  // merge: number of merges (1)
    void *scan_tmp = nullptr;       // block sums for the scans
    size_t scan_tmp_bytes = 0;
};

// Every kernel launch of the library passes its stream through counted(), so
// dem_launch_count() reports how many kernels of this library were launched
// (process-wide, all contexts); callers use it to show that the device path ran.
cudaStream_t counted(cudaStream_t s);

int dem_set_error(dem_ctx *ctx, int code, const std::string &msg);
int dem_check_cuda(dem_ctx *ctx, cudaError_t e, const char *where);
int dem_check_launch(dem_ctx *ctx, const char *where);
int dem_ensure_table(dem_ctx *ctx, int64_t table_size);
int dem_ensure_partials(dem_ctx *ctx, int splits);
int dem_ensure_sym_partials(dem_ctx *ctx, size_t bytes);
// Records a CUDA event before/after a kernel launch when profiling is on.
void dem_prof_begin(dem_ctx *ctx, const char *name, cudaStream_t s);
void dem_prof_end(dem_ctx *ctx, cudaStream_t s);

// ---------------------------------------------------------------------------
// Arithmetic shared with the oracle's restatement of the reference kernels.
// ---------------------------------------------------------------------------
// Taichi lowers x**k (integer literal k) by exponentiation by squaring.
DEM_HD double ipow3(double x) { return x * (x * x); }
DEM_HD double ipow7(double x) {
    const double x2 = x * x;
    return (x * x2) * (x2 * x2);
}
// Minimum image, direct_droplet_force_calculator.py:234-240:
// if |d| > L/2: d -= sign(d) * L
DEM_HD double mic64(double d, double L, double halfL) {
    return fabs(d) > halfL ? d - copysign(L, d) : d;
}
// numpy float remainder (npy_divmod) for a positive modulus
__device__ __forceinline__ double np_remainder(double a, double b) {
    double mod = fmod(a, b);
    if (mod != 0.0) {
        if ((b < 0) != (mod < 0)) mod += b;
    } else {
        mod = copysign(0.0, b);
    }
    return mod;
}

__device__ __forceinline__ void raise_device_error(uint32_t *err, uint32_t bit) {
    if (err) atomicOr(err, bit);
}

static inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
