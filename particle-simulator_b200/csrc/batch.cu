// batch.cu -- ensembles of independent periodic boxes stepped together.
//
// main_multi.py runs one direct simulation after another (one
// DirectDropletForceCalculator + EulerDropletSolver per initial state, no
// collision detector, main_multi.py:52-77).  Here the boxes of an ensemble
// share one set of launches per pass: the block pairs of every box form one
// work list of the symmetric pair kernel (sym.cuh), walked by a persistent
// grid, and one Euler launch moves every droplet with its own box's side.
// A step can be recorded once as a CUDA graph and replayed.  The tile shape
// (i per thread, hence the block size) and the grid (one CTA per block pair
// or a persistent grid of a multiple of the resident CTA slots) are chosen by
// timing the candidates on the ensemble itself (dem_batch_autotune).
#include <algorithm>
#include <vector>

#include "sym.cuh"

namespace dem {
int launch_euler_direct_boxes(dem_ctx *ctx, int n, int nbox, const int *off, const double *Lb, const double *x,
                              const double *y, const double *z, const double *r, const double *fx, const double *fy,
                              const double *fz, const double *vx, const double *vy, const double *vz, double stokes,
                              double dt, int periodic, double *xo, double *yo, double *zo, cudaStream_t s);
}  // namespace dem

void dem_count_launches(unsigned long long k);

using namespace dem;

namespace {
struct BoxTab {
    int B = 0;
    int *poff = nullptr, *ioff = nullptr;  // device [nbox + 1]
    int npad = 0, items = 0;
};
}  // namespace

struct dem_batch {
    dem_ctx *ctx = nullptr;
    int nbox = 0, n = 0, periodic = 1;
    std::vector<int> off_host;
    std::vector<double> L_host;
    int *off = nullptr;                    // device [nbox + 1]
    double *L = nullptr;                   // device [nbox]
    unsigned long long *scales = nullptr;  // device [nbox][2]
    BoxTab tab[2];                         // i per thread 2 and 4
    double *work = nullptr;
    int ipt = 4, ctas = 0;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long graph_kernels = 0;
};

static BoxTab &tab_for(dem_batch *b, int ipt) { return b->tab[ipt >= 4 ? 1 : 0]; }

static SymBoxes view(dem_batch *b, int ipt) {
    const BoxTab &t = tab_for(b, ipt);
    SymBoxes v{};
    v.nbox = b->nbox;
    v.n_total = b->n;
    v.npad_total = t.npad;
    v.items_total = t.items;
    v.n1 = b->n;
    v.npad1 = t.npad;
    v.L1 = b->L_host.empty() ? 1.0 : b->L_host[0];
    v.scales1 = b->scales;
    v.off = b->off;
    v.poff = t.poff;
    v.ioff = t.ioff;
    v.L = b->L;
    v.scales = b->scales;
    return v;
}

static MixedArgs fp64_args(dem_batch *b, const double *x, const double *y, const double *z, const double *r,
                           const double *fx, const double *fy, const double *fz) {
    MixedArgs m{};
    m.n = b->n;
    m.x = x;
    m.y = y;
    m.z = z;
    m.r = r;
    m.fx = fx;
    m.fy = fy;
    m.fz = fz;
    m.L = b->L_host.empty() ? 1.0 : b->L_host[0];
    m.halfL = 0.5 * m.L;
    m.scales = b->scales;
    m.err = b->ctx->d_err;
    return m;
}

static void free_batch(dem_batch *b) {
    cudaSetDevice(b->ctx->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    void *ptrs[] = {b->off, b->L, b->scales, b->work, b->tab[0].poff, b->tab[0].ioff, b->tab[1].poff, b->tab[1].ioff};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    delete b;
}

static int batch_forces(dem_batch *b, const double *x, const double *y, const double *z, const double *r,
                        double m_const, double *fx, double *fy, double *fz, cudaStream_t s) {
    dem_ctx *ctx = b->ctx;
    const SymBoxes t = view(b, b->ipt);
    int rc = dem_check_cuda(ctx, cudaMemsetAsync(b->scales, 0, 2 * sizeof(unsigned long long) * b->nbox, s), "memset");
    if (rc) return rc;
    if ((rc = launch_maxabs_boxes(ctx, t, r, nullptr, nullptr, b->scales, 0, s))) return rc;
    const MixedArgs m = fp64_args(b, x, y, z, r, nullptr, nullptr, nullptr);
    return run_sym_boxes<true>(ctx, t, b->ipt, b->ctas, b->periodic != 0, m, b->work, m_const, fx, fy, fz, s);
}

static int batch_convection(dem_batch *b, const double *x, const double *y, const double *z, const double *r,
                            const double *fx, const double *fy, const double *fz, double eta, double *vx, double *vy,
                            double *vz, cudaStream_t s) {
    dem_ctx *ctx = b->ctx;
    const SymBoxes t = view(b, b->ipt);
    int rc = dem_check_cuda(ctx, cudaMemsetAsync(b->scales, 0, 2 * sizeof(unsigned long long) * b->nbox, s), "memset");
    if (rc) return rc;
    if ((rc = launch_maxabs_boxes(ctx, t, r, nullptr, nullptr, b->scales, 0, s))) return rc;
    if ((rc = launch_maxabs_boxes(ctx, t, fx, fy, fz, b->scales, 1, s))) return rc;
    const MixedArgs m = fp64_args(b, x, y, z, r, fx, fy, fz);
    return run_sym_boxes<false>(ctx, t, b->ipt, b->ctas, b->periodic != 0, m, b->work, eta, vx, vy, vz, s);
}

static int batch_step(dem_batch *b, double *x, double *y, double *z, const double *r, double m_const, double eta,
                      double stokes, double dt, double *fx, double *fy, double *fz, double *vx, double *vy,
                      double *vz, cudaStream_t s) {
    int rc = batch_forces(b, x, y, z, r, m_const, fx, fy, fz, s);
    if (rc) return rc;
    b->ctx->sym_reuse_order = true;  // the same positions: the force pass's Morton order holds
    rc = batch_convection(b, x, y, z, r, fx, fy, fz, eta, vx, vy, vz, s);
    b->ctx->sym_reuse_order = false;
    if (rc) return rc;
    return launch_euler_direct_boxes(b->ctx, b->n, b->nbox, b->off, b->L, x, y, z, r, fx, fy, fz, vx, vy, vz, stokes,
                                     dt, b->periodic, x, y, z, s);
}

extern "C" {

int dem_batch_create(dem_ctx *ctx, int nbox, const int64_t *offsets, const double *L, int periodic, dem_batch **out) {
    if (!ctx || !out || nbox < 1 || !offsets || !L) return dem_set_error(ctx, DEM_E_INVALID, "batch: bad arguments");
    *out = nullptr;
    if (offsets[0] != 0) return dem_set_error(ctx, DEM_E_INVALID, "batch: offsets[0] must be 0");
    for (int i = 0; i < nbox; ++i) {
        if (offsets[i + 1] < offsets[i]) return dem_set_error(ctx, DEM_E_INVALID, "batch: offsets must not decrease");
        if (!(L[i] > 0.0)) return dem_set_error(ctx, DEM_E_INVALID, "batch: box sides must be positive");
    }
    if (offsets[nbox] > 0x7fffffffLL) return dem_set_error(ctx, DEM_E_CAPACITY, "batch: too many droplets");
    int rc = dem_check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (rc) return rc;
    dem_batch *b = new dem_batch();
    b->ctx = ctx;
    b->nbox = nbox;
    b->n = (int)offsets[nbox];
    b->periodic = periodic ? 1 : 0;
    b->off_host.assign(offsets, offsets + nbox + 1);
    b->L_host.assign(L, L + nbox);
    size_t work = 0;
    for (int k = 0; k < 2; ++k) {
        BoxTab &t = b->tab[k];
        t.B = SYM_T * (k ? 4 : 2);
        std::vector<int> poff(nbox + 1), ioff(nbox + 1);
        long long np = 0, it = 0;
        for (int i = 0; i < nbox; ++i) {
            poff[i] = (int)np;
            ioff[i] = (int)it;
            const long long nb = (b->off_host[i + 1] - b->off_host[i] + t.B - 1) / t.B;
            np += nb * t.B;
            it += nb * (nb + 1) / 2;
            if (np > 0x7fffffffLL || it > 0x7fffffffLL) {
                free_batch(b);
                return dem_set_error(ctx, DEM_E_CAPACITY, "batch: too many blocks");
            }
        }
        poff[nbox] = (int)np;
        ioff[nbox] = (int)it;
        t.npad = (int)np;
        t.items = (int)it;
        work = std::max(work, sym_workspace_bytes(np, it, t.B) + sym_sorted_extra_bytes(b->n, np, it, t.B));
        if ((rc = dem_check_cuda(ctx, cudaMalloc((void **)&t.poff, sizeof(int) * (nbox + 1)), "batch tables")) ||
            (rc = dem_check_cuda(ctx, cudaMalloc((void **)&t.ioff, sizeof(int) * (nbox + 1)), "batch tables")) ||
            (rc = dem_check_cuda(ctx, cudaMemcpy(t.poff, poff.data(), sizeof(int) * (nbox + 1), cudaMemcpyHostToDevice),
                                 "batch tables")) ||
            (rc = dem_check_cuda(ctx, cudaMemcpy(t.ioff, ioff.data(), sizeof(int) * (nbox + 1), cudaMemcpyHostToDevice),
                                 "batch tables"))) {
            free_batch(b);
            return rc;
        }
    }
    std::vector<int> off32(b->off_host.begin(), b->off_host.end());
    if ((rc = dem_check_cuda(ctx, cudaMalloc((void **)&b->off, sizeof(int) * (nbox + 1)), "batch tables")) ||
        (rc = dem_check_cuda(ctx, cudaMalloc((void **)&b->L, sizeof(double) * nbox), "batch tables")) ||
        (rc = dem_check_cuda(ctx, cudaMalloc((void **)&b->scales, 2 * sizeof(unsigned long long) * nbox), "batch")) ||
        (rc = dem_check_cuda(ctx, cudaMalloc((void **)&b->work, work > 0 ? work : 256), "batch workspace")) ||
        (rc = dem_check_cuda(ctx, cudaMemcpy(b->off, off32.data(), sizeof(int) * (nbox + 1), cudaMemcpyHostToDevice),
                             "batch tables")) ||
        (rc = dem_check_cuda(ctx, cudaMemcpy(b->L, L, sizeof(double) * nbox, cudaMemcpyHostToDevice), "batch tables")) ||
        (rc = dem_check_cuda(ctx, cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking), "batch stream"))) {
        free_batch(b);
        return rc;
    }
    *out = b;
    return DEM_OK;
}

void dem_batch_destroy(dem_batch *b) {
    if (b) free_batch(b);
}

int dem_batch_info(const dem_batch *b, int *nbox, int *n, int *items_ipt2, int *items_ipt4) {
    if (!b) return DEM_E_INVALID;
    if (nbox) *nbox = b->nbox;
    if (n) *n = b->n;
    if (items_ipt2) *items_ipt2 = b->tab[0].items;
    if (items_ipt4) *items_ipt4 = b->tab[1].items;
    return DEM_OK;
}

int dem_batch_set_tuning(dem_batch *b, int i_per_thread, int ctas) {
    if (!b || (i_per_thread != 2 && i_per_thread != 4) || ctas < 0)
        return dem_set_error(b ? b->ctx : nullptr, DEM_E_INVALID, "batch tuning: i_per_thread 2 or 4, ctas >= 0");
    b->ipt = i_per_thread;
    b->ctas = ctas;
    return DEM_OK;
}

int dem_batch_get_tuning(const dem_batch *b, int *i_per_thread, int *ctas) {
    if (!b) return DEM_E_INVALID;
    if (i_per_thread) *i_per_thread = b->ipt;
    if (ctas) *ctas = b->ctas;
    return DEM_OK;
}

int dem_batch_forces(dem_batch *b, const double *x, const double *y, const double *z, const double *r,
                     double m_const, double *fx, double *fy, double *fz, void *stream) {
    if (!b) return DEM_E_INVALID;
    return batch_forces(b, x, y, z, r, m_const, fx, fy, fz, (cudaStream_t)stream);
}

int dem_batch_convection(dem_batch *b, const double *x, const double *y, const double *z, const double *r,
                         const double *fx, const double *fy, const double *fz, double eta_const, double *vx,
                         double *vy, double *vz, void *stream) {
    if (!b) return DEM_E_INVALID;
    return batch_convection(b, x, y, z, r, fx, fy, fz, eta_const, vx, vy, vz, (cudaStream_t)stream);
}

int dem_batch_step(dem_batch *b, double *x, double *y, double *z, const double *r, double m_const, double eta_const,
                   double stokes_factor, double dt, double *fx, double *fy, double *fz, double *vx, double *vy,
                   double *vz, void *stream) {
    if (!b) return DEM_E_INVALID;
    return batch_step(b, x, y, z, r, m_const, eta_const, stokes_factor, dt, fx, fy, fz, vx, vy, vz,
                      (cudaStream_t)stream);
}

int dem_batch_autotune(dem_batch *b, const double *x, const double *y, const double *z, const double *r,
                       double m_const, double eta_const, double *fx, double *fy, double *fz, double *vx, double *vy,
                       double *vz, int reps, void *stream, double *best_ms) {
    if (!b || reps < 1) return DEM_E_INVALID;
    dem_ctx *ctx = b->ctx;
    cudaStream_t s = (cudaStream_t)stream;
    const bool prof = ctx->prof_enabled;
    ctx->prof_enabled = false;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int best_ipt = b->ipt, best_ctas = b->ctas;
    int rc = DEM_OK;
    for (int ipt : {2, 4}) {
        const int slots = sym_resident_ctas(ipt, b->periodic != 0, true) * ctx->sm_count;
        for (int ctas : {0, slots, 2 * slots, 4 * slots}) {
            if (ctas > 0 && ctas >= tab_for(b, ipt).items) continue;  // same as one CTA per item
            b->ipt = ipt;
            b->ctas = ctas;
            for (int w = 0; w < 1 + reps && !rc; ++w) {
                if (w == 1) cudaEventRecord(e0, s);
                rc = batch_forces(b, x, y, z, r, m_const, fx, fy, fz, s);
                if (!rc) rc = batch_convection(b, x, y, z, r, fx, fy, fz, eta_const, vx, vy, vz, s);
            }
            cudaEventRecord(e1, s);
            if (!rc) rc = dem_check_cuda(ctx, cudaEventSynchronize(e1), "autotune");
            if (rc) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms / reps < best) {
                best = ms / reps;
                best_ipt = ipt;
                best_ctas = ctas;
            }
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->prof_enabled = prof;
    b->ipt = best_ipt;
    b->ctas = best_ctas;
    if (best_ms) *best_ms = best;
    return rc;
}

int dem_batch_capture(dem_batch *b, double *x, double *y, double *z, const double *r, double m_const,
                      double eta_const, double stokes_factor, double dt, double *fx, double *fy, double *fz,
                      double *vx, double *vy, double *vz) {
    if (!b) return DEM_E_INVALID;
    dem_ctx *ctx = b->ctx;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    const bool prof = ctx->prof_enabled;
    ctx->prof_enabled = false;  // no timing events inside the graph
    const unsigned long long k0 = dem_launch_count();
    int rc = dem_check_cuda(ctx, cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal), "capture");
    int rc2 = DEM_OK;
    if (!rc) {
        rc2 = batch_step(b, x, y, z, r, m_const, eta_const, stokes_factor, dt, fx, fy, fz, vx, vy, vz, b->cap_stream);
        rc = dem_check_cuda(ctx, cudaStreamEndCapture(b->cap_stream, &b->graph), "capture");
    }
    ctx->prof_enabled = prof;
    if (rc2) return rc2;
    if (rc) return rc;
    b->graph_kernels = dem_launch_count() - k0;
    return dem_check_cuda(ctx, cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
}

int dem_batch_replay(dem_batch *b, int steps, void *stream) {
    if (!b || steps < 0) return DEM_E_INVALID;
    if (!b->exec) return dem_set_error(b->ctx, DEM_E_NOT_ALLOCATED, "batch: no captured step");
    for (int i = 0; i < steps; ++i) {
        int rc = dem_check_cuda(b->ctx, cudaGraphLaunch(b->exec, (cudaStream_t)stream), "graph launch");
        if (rc) return rc;
        dem_count_launches(b->graph_kernels);
    }
    return DEM_OK;
}

}  // extern "C"
