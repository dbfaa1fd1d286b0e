// ctx.cu -- context, workspace and error handling of libdem_b200.
#include <atomic>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "scan.cuh"

#define DEM_VERSION "dem_b200 0.1 (sm_100a)"

static std::atomic<unsigned long long> g_launches{0};

cudaStream_t counted(cudaStream_t s) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return s;
}

unsigned long long dem_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

// Kernels launched by a CUDA graph replay (they bypass counted()).
void dem_count_launches(unsigned long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

extern "C" void dem_count_replayed_launches(unsigned long long k) { dem_count_launches(k); }

namespace dem {
int sym_sorted_prepare(dem_ctx *ctx);
int direct_plan(const dem_ctx *ctx, int n, int periodic, int *schedule, int *i_per_thread, int *threads,
                long long *ctas, int *j_splits);
}

int dem_set_error(dem_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

int dem_check_cuda(dem_ctx *ctx, cudaError_t e, const char *where) {
    if (e == cudaSuccess) return DEM_OK;
    return dem_set_error(ctx, DEM_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

int dem_check_launch(dem_ctx *ctx, const char *where) { return dem_check_cuda(ctx, cudaGetLastError(), where); }

template <typename T>
static int grow(dem_ctx *ctx, T **p, size_t count, const char *what) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    return dem_check_cuda(ctx, cudaMalloc((void **)p, sizeof(T) * (count > 0 ? count : 1)), what);
}

int dem_ensure_table(dem_ctx *ctx, int64_t table_size) {
    if (table_size <= ctx->table_capacity) return DEM_OK;
    int rc;
    if ((rc = grow(ctx, &ctx->bucket_count, (size_t)table_size, "hash table"))) return rc;
    if ((rc = grow(ctx, &ctx->bucket_start, (size_t)table_size + 1, "hash table"))) return rc;
    if ((rc = grow(ctx, &ctx->bucket_cursor, (size_t)table_size, "hash table"))) return rc;
    ctx->table_capacity = table_size;
    return DEM_OK;
}

int dem_ensure_partials(dem_ctx *ctx, int splits) {
    if (splits <= ctx->partial_splits) return DEM_OK;
    int rc = grow(ctx, &ctx->partial, (size_t)splits * 3 * (size_t)ctx->capacity, "partial sums");
    if (rc) return rc;
    ctx->partial_splits = splits;
    return DEM_OK;
}

int dem_ensure_sym_partials(dem_ctx *ctx, size_t bytes) {
    if (bytes <= ctx->sym_partial_bytes) return DEM_OK;
    ctx->sym_partial_bytes = 0;
    int rc = grow(ctx, &ctx->sym_partial, bytes / sizeof(double) + 1, "symmetric partial sums");
    if (rc) return rc;
    ctx->sym_partial_bytes = bytes;
    return DEM_OK;
}

static cudaEvent_t prof_event(dem_ctx *ctx) {
    if (!ctx->prof_pool.empty()) {
        cudaEvent_t e = ctx->prof_pool.back();
        ctx->prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void dem_prof_begin(dem_ctx *ctx, const char *name, cudaStream_t s) {
    if (!ctx->prof_enabled) return;
    dem_prof_rec r{name, prof_event(ctx), prof_event(ctx)};
    cudaEventRecord(r.start, s);
    ctx->prof.push_back(r);
}

void dem_prof_end(dem_ctx *ctx, cudaStream_t s) {
    if (!ctx->prof_enabled || ctx->prof.empty()) return;
    cudaEventRecord(ctx->prof.back().stop, s);
}

static void prof_clear(dem_ctx *ctx) {
    for (auto &r : ctx->prof) {
        ctx->prof_pool.push_back(r.start);
        ctx->prof_pool.push_back(r.stop);
    }
    ctx->prof.clear();
}

namespace {
// An empty kernel of this library: the runtime reports the binary version of
// the code it would load for it, i.e. the architecture the library was built for.
__global__ void binary_version_probe_kernel() {}
}  // namespace

extern "C" {

const char *dem_version(void) { return DEM_VERSION; }

int dem_kernel_binary_version(int device, int *version) {
    if (!version) return DEM_E_INVALID;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return DEM_E_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return DEM_E_CUDA;
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, binary_version_probe_kernel);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return DEM_E_CUDA;
    }
    *version = a.binaryVersion;
    return DEM_OK;
}

int dem_profile_enable(dem_ctx *ctx, int enable) {
    if (!ctx) return DEM_E_INVALID;
    ctx->prof_enabled = enable != 0;
    prof_clear(ctx);
    return DEM_OK;
}

int dem_profile_read(dem_ctx *ctx, const char *name, double *total_ms, int *launches) {
    if (!ctx || !name || !total_ms || !launches) return DEM_E_INVALID;
    double ms = 0.0;
    int k = 0;
    for (auto &r : ctx->prof) {
        if (strcmp(r.name, name) != 0) continue;
        int rc = dem_check_cuda(ctx, cudaEventSynchronize(r.stop), "profile");
        if (rc) return rc;
        float t = 0.f;
        rc = dem_check_cuda(ctx, cudaEventElapsedTime(&t, r.start, r.stop), "profile");
        if (rc) return rc;
        ms += t;
        ++k;
    }
    *total_ms = ms;
    *launches = k;
    return DEM_OK;
}

int dem_profile_reset(dem_ctx *ctx) {
    if (!ctx) return DEM_E_INVALID;
    for (auto &r : ctx->prof) cudaEventSynchronize(r.stop);
    prof_clear(ctx);
    return DEM_OK;
}

int dem_ctx_reserve(dem_ctx *ctx, int capacity) {
    if (!ctx) return DEM_E_INVALID;
    if (capacity < 1) capacity = 1;
    if (capacity <= ctx->capacity) return DEM_OK;
    int rc = dem_check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (rc) return rc;
    const size_t n = (size_t)capacity;
    if ((rc = grow(ctx, &ctx->pack_a, n, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->pack_b, n, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->cell_hash, n, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->cell_xyz, 3 * n, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->sorted_idx, n, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->hash_pos, 2 * n, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->hash_pos32, n, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->pair_count, n + 1, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->pair_offset, n + 1, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->flags, n + 1, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->keep_off, n + 1, "workspace"))) return rc;
    if ((rc = grow(ctx, &ctx->merged_buf, 4 * n, "workspace"))) return rc;
    ctx->capacity = capacity;
    // partial sums depend on capacity: re-size lazily
    if (ctx->partial) cudaFree(ctx->partial);
    ctx->partial = nullptr;
    ctx->partial_splits = 0;
    return DEM_OK;
}

int dem_ctx_create(int device, int capacity, dem_ctx **out) {
    if (!out) return DEM_E_INVALID;
    *out = nullptr;
    dem_ctx *ctx = new dem_ctx();
    ctx->device = device;
    int rc = dem_check_cuda(ctx, cudaSetDevice(device), "cudaSetDevice");
    if (!rc) rc = dem_check_cuda(ctx, cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device),
                                 "cudaDeviceGetAttribute");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&ctx->d_err, sizeof(uint32_t)), "error word");
    if (!rc) rc = dem_check_cuda(ctx, cudaMemset(ctx->d_err, 0, sizeof(uint32_t)), "error word");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&ctx->dscratch, 8 * sizeof(double)), "scratch");
    if (!rc) rc = dem_check_cuda(ctx, cudaMalloc((void **)&ctx->merged_cnt, 4 * sizeof(int32_t)), "scratch");
    if (!rc) rc = dem_ctx_reserve(ctx, capacity);
    // scan block sums (fixed size) and the sorted pair kernels' shared-memory limit, set up front so
    // that no later call allocates or changes a kernel attribute (calls may run under stream capture)
    if (!rc) {
        const size_t need = sizeof(int64_t) * (dem::SCAN_MAX_BLOCKS + 1);
        rc = dem_check_cuda(ctx, cudaMalloc(&ctx->scan_tmp, need), "scan workspace");
        if (!rc) ctx->scan_tmp_bytes = need;
    }
    if (!rc) rc = dem::sym_sorted_prepare(ctx);
    if (rc) {
        fprintf(stderr, "dem_ctx_create: %s\n", ctx->last_error.c_str());
        dem_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return DEM_OK;
}

void dem_ctx_destroy(dem_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    void *ptrs[] = {ctx->d_err,         ctx->pack_a,      ctx->pack_b,     ctx->partial,    ctx->dscratch,
                    ctx->cell_hash,     ctx->cell_xyz, ctx->bucket_count, ctx->bucket_start, ctx->bucket_cursor, ctx->sorted_idx, ctx->hash_pos, ctx->hash_pos32,
                    ctx->pair_count,    ctx->pair_offset, ctx->flags,      ctx->keep_off,   ctx->merged_buf,
                    ctx->merged_cnt,    ctx->scan_tmp,    ctx->sym_partial};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    prof_clear(ctx);
    for (cudaEvent_t e : ctx->prof_pool) cudaEventDestroy(e);
    delete ctx;
}

int dem_ctx_capacity(const dem_ctx *ctx) { return ctx ? ctx->capacity : 0; }

const char *dem_last_error(const dem_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int dem_device_errors(dem_ctx *ctx, uint32_t *flags_host, void *stream) {
    if (!ctx || !flags_host) return DEM_E_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = dem_check_cuda(ctx, cudaMemcpyAsync(flags_host, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                            "read error word");
    if (!rc) rc = dem_check_cuda(ctx, cudaStreamSynchronize(s), "read error word");
    if (!rc) rc = dem_check_cuda(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), s), "clear error word");
    return rc;
}

int dem_direct_set_tuning(dem_ctx *ctx, int i_per_thread, int threads, int j_splits, double near_force,
                          double near_oseen, int schedule) {
    if (!ctx) return DEM_E_INVALID;
    if (i_per_thread) {
        if (i_per_thread != 1 && i_per_thread != 2 && i_per_thread != 4 && i_per_thread != 8)
            return dem_set_error(ctx, DEM_E_INVALID, "i_per_thread must be 1, 2, 4 or 8");
        ctx->tuning.i_per_thread = i_per_thread;
    }
    if (threads) {
        if (threads < 64 || threads > 512 || threads % 32)
            return dem_set_error(ctx, DEM_E_INVALID, "threads must be a multiple of 32 in [64, 512]");
        ctx->tuning.threads = threads;
    }
    if (j_splits < 0) return dem_set_error(ctx, DEM_E_INVALID, "j_splits must be >= 0");
    ctx->tuning.j_splits = j_splits;
    if (near_force > 0) ctx->tuning.near_force = near_force;
    if (near_oseen > 0) ctx->tuning.near_oseen = near_oseen;
    if (schedule < DEM_SCHED_AUTO || schedule > DEM_SCHED_SYMMETRIC_PLAIN)
        return dem_set_error(ctx, DEM_E_INVALID, "unknown schedule");
    ctx->tuning.schedule = schedule;
    return DEM_OK;
}

int dem_direct_get_tuning(const dem_ctx *ctx, int *i_per_thread, int *threads, int *j_splits, double *near_force,
                          double *near_oseen, int *schedule) {
    if (!ctx) return DEM_E_INVALID;
    if (i_per_thread) *i_per_thread = ctx->tuning.i_per_thread;
    if (threads) *threads = ctx->tuning.threads;
    if (j_splits) *j_splits = ctx->tuning.j_splits;
    if (near_force) *near_force = ctx->tuning.near_force;
    if (near_oseen) *near_oseen = ctx->tuning.near_oseen;
    if (schedule) *schedule = ctx->tuning.schedule;
    return DEM_OK;
}

int dem_direct_plan(const dem_ctx *ctx, int n, int periodic, int *schedule, int *i_per_thread, int *threads,
                    long long *ctas, int *j_splits) {
    if (!ctx || n < 0 || !schedule || !i_per_thread || !threads || !ctas || !j_splits) return DEM_E_INVALID;
    return dem::direct_plan(ctx, n, periodic, schedule, i_per_thread, threads, ctas, j_splits);
}

}  // extern "C"
