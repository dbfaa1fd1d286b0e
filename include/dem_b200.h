/*
 * dem_b200.h -- C ABI of libdem_b200.so, the B200 (sm_100a) implementation of
 * the DEM droplet hot path of ddkx21/particle-simulator.
 *
 * Conventions
 *   - Every array argument is a DEVICE pointer (cudaMalloc'd or a torch CUDA
 *     tensor's data_ptr()), except where a comment says "host".
 *   - Positions, forces and velocities are structure-of-arrays: one double
 *     array per Cartesian component, length n.  Radii: double[n].
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Calls are asynchronous with respect to the host unless the
 *     comment says the call synchronises.
 *   - Return value: DEM_OK or one of the DEM_E_* codes; dem_last_error()
 *     gives the message.  The Python layer maps DEM_E_CAPACITY and
 *     DEM_E_INVALID to ValueError and DEM_E_NOT_ALLOCATED to RuntimeError,
 *     the exception types the reference raises.
 *   - One context per stream; a context is not shared between host threads.
 *
 * Each entry point names the reference function it replaces (path:line in
 * ddkx21/particle-simulator).
 */
#ifndef DEM_B200_H
#define DEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define DEM_API __attribute__((visibility("default")))
#else
#define DEM_API
#endif

#define DEM_OK 0
#define DEM_E_INVALID 1       /* bad argument                                   */
#define DEM_E_CAPACITY 2      /* n (or a pair/node count) exceeds a capacity    */
#define DEM_E_CUDA 3          /* CUDA runtime error                             */
#define DEM_E_DEVICE 4        /* a kernel raised a device error flag            */
#define DEM_E_NOT_ALLOCATED 5 /* optional data not allocated                    */

/* precision of the direct O(N^2) passes */
#define DEM_PREC_FP64 0  /* reference drop-in: bit-exact with the reference expression order */
#define DEM_PREC_MIXED 1 /* FP32 pair terms, compensated sums, FP64 near-contact pairs       */

/* device error flags (dem_device_errors) */
#define DEM_DEVERR_WAIT_TIMEOUT 1u  /* a bounded wait (mbarrier / flag) ran out   */
#define DEM_DEVERR_PAIR_OVERFLOW 2u /* more colliding pairs than the pair buffer  */
#define DEM_DEVERR_NODE_OVERFLOW 4u /* octree node pool exhausted                 */
#define DEM_DEVERR_NONFINITE 8u     /* a non-finite value was produced            */

typedef struct dem_ctx dem_ctx;
typedef struct dem_corr dem_corr; /* periodic-image correction grid (dem_corr_create) */

/* ---- context --------------------------------------------------------- */
/* Creates a context on `device` with room for `capacity` particles.
 * Replaces the per-class Taichi field allocation of
 * dem/force_calculator/direct_droplet_force_calculator.py:37-48 and
 * dem/collision_detector/spatial_hash_collision_detector.py:45-69. */
DEM_API int dem_ctx_create(int device, int capacity, dem_ctx **out);
DEM_API void dem_ctx_destroy(dem_ctx *ctx);
/* Grows the workspace to `capacity` particles (no-op when already large enough). */
DEM_API int dem_ctx_reserve(dem_ctx *ctx, int capacity);
DEM_API int dem_ctx_capacity(const dem_ctx *ctx);
DEM_API const char *dem_last_error(const dem_ctx *ctx);
/* Reads and clears the device error flags (DEM_DEVERR_*).  Synchronises `stream`. */
DEM_API int dem_device_errors(dem_ctx *ctx, uint32_t *flags_host, void *stream);
/* Library version string (host). */
DEM_API const char *dem_version(void);
/* The binary version (major * 10 + minor, 100 for sm_100a) of the device code
 * the CUDA runtime loads for this library's kernels on `device`, from
 * cudaFuncGetAttributes.  Needs a CUDA device.  No reference counterpart. */
DEM_API int dem_kernel_binary_version(int device, int *version);
/* Number of kernels this library has launched in the process so far (all
 * contexts and devices; host-side counter, no synchronisation).  The
 * difference across a region is the count of the library's launches in it. */
DEM_API unsigned long long dem_launch_count(void);
/* Adds k to that counter: kernels of this library replayed from a CUDA graph
 * that the caller captured (a replay does not pass through the library). */
DEM_API void dem_count_replayed_launches(unsigned long long k);

/* Opt-in kernel timing: while enabled, CUDA events are recorded on the launch
 * stream around the main kernels ("mixed_force_pass", "mixed_convection_pass",
 * "fp64_force_pass", "fp64_convection_pass", "hash_detect").
 * dem_profile_read synchronises on the recorded events and returns the summed
 * device time and the number of launches of `name`. */
DEM_API int dem_profile_enable(dem_ctx *ctx, int enable);
DEM_API int dem_profile_read(dem_ctx *ctx, const char *name, double *total_ms, int *launches);
DEM_API int dem_profile_reset(dem_ctx *ctx);

/* schedules of the mixed-precision direct passes */
#define DEM_SCHED_AUTO 0      /* symmetric when its partial sums fit, else split */
#define DEM_SCHED_SPLIT 1     /* every ordered pair; the j range split in chunks */
#define DEM_SCHED_SYMMETRIC 2 /* every unordered pair once (F_ji = -F_ij, Oseen tensor even); one box:
                                 blocks of droplets in Morton order, far j's without the per-pair
                                 minimum image and tests */
#define DEM_SCHED_SYMMETRIC_PLAIN 3 /* symmetric, blocks in the caller's droplet order (every pair takes the
                                       minimum image and the tests) */

/* Tuning of the mixed-precision direct kernels (0 keeps the current value).
 *   i_per_thread  i-particles register-blocked per thread (1, 2, 4 or 8;
 *                 the symmetric schedule uses 1, 2 or 4)
 *   threads       threads per CTA of the split schedule (64..512, multiple of 32)
 *   j_splits      number of j-chunks of the split schedule (>=1; 0 = auto)
 *   near_force    FP64 radius factor k: pairs with |r_ij| <= k (r_i + r_j) are
 *   near_oseen    computed in FP64 (force / convection pass)
 *   schedule      DEM_SCHED_* (this one is always applied) */
DEM_API int dem_direct_set_tuning(dem_ctx *ctx, int i_per_thread, int threads, int j_splits, double near_force,
                                  double near_oseen, int schedule);
DEM_API int dem_direct_get_tuning(const dem_ctx *ctx, int *i_per_thread, int *threads, int *j_splits,
                                  double *near_force, double *near_oseen, int *schedule);
/* The plan the mixed-precision passes run for n droplets under the current
 * tuning (no launch): the resolved schedule (DEM_SCHED_SPLIT,
 * DEM_SCHED_SYMMETRIC or DEM_SCHED_SYMMETRIC_PLAIN), i-per-thread blocking,
 * threads per CTA, CTAs per pass
 * and, for the split schedule, the number of j-chunks. */
DEM_API int dem_direct_plan(const dem_ctx *ctx, int n, int periodic, int *schedule, int *i_per_thread,
                            int *threads, long long *ctas, int *j_splits);

/* ---- Barnes-Hut octree from Morton keys (fast form) ------------------- */
/* The Barnes-Hut method of dem/octree (flat_tree.py:180-1588) built from
 * 30-bit Morton keys: positions -> keys in the root cube ([0, L)^3 when
 * periodic, else the droplets' bounding cube) -> stable on-device radix sort
 * -> octree level by level from key prefixes (a node holding more than
 * leaf_size droplets is split into its non-empty octants, at most 10 levels)
 * -> R^3 sums and R^3-weighted centres.  Walks use the reference's acceptance
 * test s^2 < theta^2 D^2 (flat_tree.py:871), opened per warp of 32 spatially
 * adjacent targets, with monopole forces (:873-884), Stokeslet + dipole
 * velocities (:1215-1265) and exact leaf pairs with the contact cut
 * r^2 >= (r_i + r_j)^2 (:835).  A leaf pair's separation is the FP64
 * minimum-image vector from the target to the leaf centre (once per leaf
 * visit) plus the source's FP32 offset from that centre, recomputed in FP64
 * when a component lies within 1e-6 L of L/2; node separations and all terms
 * are FP32.  Results
 * approximate the direct sums; the FP64 reference-parity tree is dem_tree_*.
 * dem_bh_build synchronises `stream` once per tree level (level sizes). */
typedef struct dem_bh dem_bh;
DEM_API int dem_bh_create(dem_ctx *ctx, int capacity, dem_bh **out);
DEM_API void dem_bh_destroy(dem_bh *bh);
DEM_API int dem_bh_build(dem_bh *bh, int n, const double *x, const double *y, const double *z, const double *r,
                         double L, int periodic, int leaf_size, void *stream);
/* Dipole forces of the built tree's droplets, in the caller's order. */
DEM_API int dem_bh_forces(dem_bh *bh, double m_const, double theta, double *fx, double *fy, double *fz, void *stream);
/* Oseen convection from the tree (f* = NULL: the forces of the last
 * dem_bh_forces); with stokes_factor > 0 the total velocity
 * F / (stokes_factor r) + V (flat_tree.py:1326-1347), else V alone. */
DEM_API int dem_bh_velocity(dem_bh *bh, const double *fx, const double *fy, const double *fz, double eta_const,
                            double theta, double stokes_factor, double *vx, double *vy, double *vz, void *stream);
/* Periodic boxes: a node whose cell is larger than L / 2^window_level is
 * opened unless the whole cell lies inside the target's minimum-image window
 * (|D_axis| + s < L/2); smaller straddling cells are taken at their centre's
 * image, as the reference does for every node (flat_tree.py:871).
 * 0 (the default) = the reference's rule. */
DEM_API int dem_bh_set_window(dem_bh *bh, int window_level);
/* Attaches a periodic-image correction (dem_corr_create) to the velocity
 * walk, NULL detaches it: FP32 correction terms at every exact leaf pair and
 * every accepted node (at the node's R^3 centre with its force sum), and
 * the self term self_coeff * F_i when stokes_factor <= 0 (the reference's
 * walks, flat_tree.py:1070-1131, :1171-1213, :1271-1276).  The grid must
 * outlive its use by the tree. */
DEM_API int dem_bh_set_correction(dem_bh *bh, const dem_corr *corr);
/* out (host, 8): nodes, levels, droplets, node capacity, leaf pair terms and
 * accepted-node terms of the last walk (summed over targets), leaf size,
 * droplet capacity. */
DEM_API int dem_bh_stats(dem_bh *bh, int64_t *out);

/* ---- adjoint of the direct step --------------------------------------- */
/* Vector-Jacobian product of the direct-path droplet velocity
 *   u_i = F_i / (stokes_factor r_i) + V_i    (euler_droplet_solver.py:121-125)
 * with F the dipole forces (direct_droplet_force_calculator.py:183-253, contact
 * cut |d| > r_i + r_j) and V the Oseen convection of F (:354-411), in FP64.
 * Given the cotangent lambda on u (l*), returns
 *   g*_i = sum_k lambda_k . du_k/dx_i,  gr_i = sum_k lambda_k . du_k/dr_i,
 * and mu (m*), the cotangent reaching the forces:
 *   mu_i = lambda_i / (stokes_factor r_i) + eta sum_{j != i} G(x_i - x_j) lambda_j.
 * f* must hold the forces of this state (dem_direct_forces, FP64 or mixed).
 * The collision cut and the periodic wrap are treated as non-differentiable;
 * d/dE of u is 2 u / E (m_const is proportional to E^2) and needs no call. */
DEM_API int dem_direct_vjp(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                           const double *fx, const double *fy, const double *fz, const double *lx, const double *ly,
                           const double *lz, double m_const, double eta_const, double stokes_factor, double L,
                           int periodic, double *mx, double *my, double *mz, double *gx, double *gy, double *gz,
                           double *gr, void *stream);

/* ---- ensembles of independent boxes ---------------------------------- */
/* main_multi.py:52-77 runs one direct simulation per initial state, one after
 * another, without a collision detector.  A batch steps many such boxes
 * together: droplets [offsets[b], offsets[b+1]) of the caller's SoA arrays live
 * in a periodic (or open) box of side L[b]; every pass is one set of launches
 * over all boxes (the mixed-precision symmetric pair kernel walks the block
 * pairs of every box in one grid).  Per box the results are bit-identical to
 * the single-box mixed-precision calls with the same i-per-thread blocking.
 * offsets (host, nbox + 1 entries, offsets[0] = 0, non-decreasing) and L
 * (host, nbox) are copied.  The batch keeps its own workspace; it uses the
 * context's device, error word and near-pair factors. */
typedef struct dem_batch dem_batch;
DEM_API int dem_batch_create(dem_ctx *ctx, int nbox, const int64_t *offsets, const double *L, int periodic,
                             dem_batch **out);
DEM_API void dem_batch_destroy(dem_batch *batch);
/* Boxes, droplets and block pairs per pass for i-per-thread 2 and 4. */
DEM_API int dem_batch_info(const dem_batch *batch, int *nbox, int *n, int *items_ipt2, int *items_ipt4);
/* i_per_thread 2 or 4 (block size 256 / 512); ctas = 0: one CTA per block
 * pair, else a persistent grid of that many CTAs. */
DEM_API int dem_batch_set_tuning(dem_batch *batch, int i_per_thread, int ctas);
DEM_API int dem_batch_get_tuning(const dem_batch *batch, int *i_per_thread, int *ctas);
/* Forces / convection of every box (mixed precision; as dem_direct_forces and
 * dem_direct_convection per box). */
DEM_API int dem_batch_forces(dem_batch *batch, const double *x, const double *y, const double *z, const double *r,
                             double m_const, double *fx, double *fy, double *fz, void *stream);
DEM_API int dem_batch_convection(dem_batch *batch, const double *x, const double *y, const double *z,
                                 const double *r, const double *fx, const double *fy, const double *fz,
                                 double eta_const, double *vx, double *vy, double *vz, void *stream);
/* One Euler step of every box, in place (euler_droplet_solver.py:121-131 per
 * box): forces, convection, x += (F / (stokes_factor r) + v) dt, x %= L[b].
 * f* and v* receive this step's forces and convection velocities. */
DEM_API int dem_batch_step(dem_batch *batch, double *x, double *y, double *z, const double *r, double m_const,
                           double eta_const, double stokes_factor, double dt, double *fx, double *fy, double *fz,
                           double *vx, double *vy, double *vz, void *stream);
/* Times every candidate tiling (i per thread 2 / 4 x one CTA per block pair or
 * a persistent grid of 1, 2, 4 x the resident CTA slots) over `reps` force +
 * convection passes on these inputs and keeps the fastest.  Synchronises
 * `stream`; overwrites f* and v* with valid results; best_ms (host, may be
 * NULL) receives the best time per force + convection pair of passes. */
DEM_API int dem_batch_autotune(dem_batch *batch, const double *x, const double *y, const double *z, const double *r,
                               double m_const, double eta_const, double *fx, double *fy, double *fz, double *vx,
                               double *vy, double *vz, int reps, void *stream, double *best_ms);
/* Records one dem_batch_step on these buffers as a CUDA graph (nothing runs);
 * dem_batch_replay launches it `steps` times on `stream`.  The graph keeps the
 * pointers and scalars given here; a new capture replaces the old one. */
DEM_API int dem_batch_capture(dem_batch *batch, double *x, double *y, double *z, const double *r, double m_const,
                              double eta_const, double stokes_factor, double dt, double *fx, double *fy, double *fz,
                              double *vx, double *vy, double *vz);
DEM_API int dem_batch_replay(dem_batch *batch, int steps, void *stream);

/* ---- layout ---------------------------------------------------------- */
/* (n, 3) row-major <-> three component arrays.  The reference's public
 * methods take and return (N, 3) numpy arrays
 * (direct_droplet_force_calculator.py:260-305); the kernels work on SoA. */
DEM_API int dem_aos_to_soa(dem_ctx *ctx, int n, const double *aos, double *x, double *y, double *z, void *stream);
DEM_API int dem_soa_to_aos(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, double *aos,
                           void *stream);

/* ---- direct O(N^2) passes --------------------------------------------- */
/* Dipole force on every droplet.
 * Replaces DirectDropletForceCalculator._calculate_forces,
 * dem/force_calculator/direct_droplet_force_calculator.py:202-253
 * (pair term _calculate_one_force :183-200; MIC :234-240; cut r > r_i + r_j). */
DEM_API int dem_direct_forces(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                      double m_const, double L, int periodic, int precision, double *fx, double *fy, double *fz,
                      void *stream);

/* Oseen convection velocity of every droplet (correction off).  r (radii)
 * may be NULL for DEM_PREC_FP64; the mixed path uses it for its near-contact
 * test.
 * Replaces DirectDropletForceCalculator._calculate_convection_velocities,
 * dem/force_calculator/direct_droplet_force_calculator.py:354-411. */
DEM_API int dem_direct_convection(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                          const double *fx, const double *fy, const double *fz, double eta_const, double L,
                          int periodic, int precision, double *vx, double *vy, double *vz, void *stream);

/* Forces, then the Oseen convection of those forces (correction off): the
 * two calls above on the same positions, in one call.  With DEM_PREC_MIXED
 * the convection pass reuses the Morton order the force pass sorted the
 * droplets into (the results equal those of the two calls, bit for bit).
 * r may not be NULL.
 * Replaces DirectDropletForceCalculator.calculate_forces_and_convection,
 * dem/force_calculator/direct_droplet_force_calculator.py:470-527. */
DEM_API int dem_direct_forces_and_convection(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                                             const double *r, double m_const, double eta_const, double L,
                                             int periodic, int precision, double *fx, double *fy, double *fz,
                                             double *vx, double *vy, double *vz, void *stream);

/* ---- periodic-image Oseen correction (COMSOL lattice grid) ------------ */
/* A correction grid uploaded to the device.  grid_u/v/w: HOST arrays of n^3
 * doubles in C order [ix][iy][iz], the velocity of the periodic images of a
 * unit z-force on the nodes grid_min + k / inv_dx (k = 0..n-1) of every axis
 * (COMSOLLatticeCorrection.get_grid_data).  The scalars are those of
 * load_periodic_correction:
 *   Fz_inv = 1 / Fz_comsol, L_ratio = L_comsol / L_sim,
 *   eta_ratio = eta_comsol / eta_sim, self_coeff = w(0,0,0) * Fz_inv * eta_ratio * L_ratio.
 * 2 <= n <= DEM_CORR_MAX_GRID.  Device memory: 320 (n-1)^3 bytes.
 * Replaces the correction fields and load_periodic_correction of
 * dem/force_calculator/direct_droplet_force_calculator.py:56-120 and
 * dem/octree/flat_tree.py:125-167. */
#define DEM_CORR_MAX_GRID 256
DEM_API int dem_corr_create(dem_ctx *ctx, int n, const double *grid_u, const double *grid_v, const double *grid_w,
                            double grid_min, double inv_dx, double Fz_inv, double L_ratio, double eta_ratio,
                            double self_coeff, dem_corr **out);
DEM_API void dem_corr_destroy(dem_corr *corr);
/* Host scalars: grid points per axis, the per-pair factor
 * Fz_inv * eta_ratio * L_ratio, the self coefficient (NULL skips). */
DEM_API int dem_corr_info(const dem_corr *corr, int *n, double *common, double *self_coeff);

/* Roofline probe of the FP32 correction pass (no counterpart in the
 * reference): ctas x 256 threads each read per_thread cells of the FP32 table
 * at pseudo-random positions, 96 bytes per cell in three 256-bit loads, and
 * write one float each to out (device, ctas * 256 floats).  Time it on
 * `stream` to get the table's random-gather bandwidth. */
DEM_API int dem_corr_gather_probe(const dem_corr *corr, int ctas, int per_thread, float *out, void *stream);

/* Oseen convection with the periodic-image correction: as
 * dem_direct_convection, plus for every pair j != i the correction of
 * d = MIC(x_i - x_j) (three permuted trilinear lookups contracted with F_j)
 * and after the sum the self term self_coeff * F_i.  DEM_PREC_FP64 adds each
 * pair's correction right after its Stokeslet term, bit-identical to the
 * reference's order; DEM_PREC_MIXED runs the mixed Oseen pass and an FP32
 * correction pass (FP32 trilinear forms, FP64 tile sums).  corr == NULL is
 * DEM_E_NOT_ALLOCATED.
 * Replaces DirectDropletForceCalculator._calculate_convection_velocities with
 * corr_enabled == 1, dem/force_calculator/direct_droplet_force_calculator.py:354-464
 * (lookups _precompute_grid_idx / _interp_precomp :146-182). */
DEM_API int dem_direct_convection_corr(dem_ctx *ctx, const dem_corr *corr, int n, const double *x, const double *y,
                                       const double *z, const double *r, const double *fx, const double *fy,
                                       const double *fz, double eta_const, double L, int periodic, int precision,
                                       double *vx, double *vy, double *vz, void *stream);

/* Explicit Euler update of the direct path, out of place (xo may equal x):
 *   x_o = (x + (F / (stokes_factor * r) + v) * dt) mod L   (numpy remainder when periodic)
 * Replaces dem/solver/euler_droplet_solver.py:121-131. */
DEM_API int dem_euler_update(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                     const double *fx, const double *fy, const double *fz, const double *vx, const double *vy,
                     const double *vz, double stokes_factor, double dt, double L, int periodic, double *xo,
                     double *yo, double *zo, void *stream);

/* Euler update of the tree path, x_o = (x + v_total * dt) mod L.
 * Replaces dem/solver/euler_droplet_solver.py:119, :130-131. */
DEM_API int dem_euler_update_total(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                           const double *vx, const double *vy, const double *vz, double dt, double L, int periodic,
                           double *xo, double *yo, double *zo, void *stream);

/* ---- spatial hash collision detection -------------------------------- */
/* Unique colliding pairs (i < j, lexicographic order) with the reference's
 * cell/hash semantics: cell = 2 max r, grid = max(1, ceil(L / cell)), hash
 * (ix*73856093 ^ iy*19349663 ^ iz*83492791) & (table_size - 1), 27 neighbour
 * cells, MIC distance <= r_i + r_j.
 * pairs: int32[pair_capacity][2] (device).  counts: int64[2] (device):
 * counts[0] = number of unique pairs (may exceed pair_capacity: then the
 * buffer holds the lexicographically first pair_capacity pairs of the sorted
 * set and DEM_DEVERR_PAIR_OVERFLOW is raised), counts[1] = raw hits before
 * de-duplication.
 * Replaces SpatialHashCollisionDetector.detect,
 * dem/collision_detector/spatial_hash_collision_detector.py:233-316
 * (kernels :74-229, np.unique :312). */
DEM_API int dem_hash_detect(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
                    double L, int periodic, int table_size, int32_t *pairs, int64_t pair_capacity, int64_t *counts,
                    void *stream);

/* Every pair with (minimum-image when periodic) distance <= r_i + r_j, with
 * the same outputs as dem_hash_detect, but on a grid of whole cells
 * (floor(L / 2 max r) cells of side L / grid), so that no touching pair
 * across the periodic faces is skipped.  (dem_hash_detect keeps the
 * reference's grid, ceil(L / 2 max r) cells with a partial last one.)  Used by
 * the droplet generators' overlap rejection with radii inflated by half the
 * minimum gap; L > 0 also in open boxes (positions in [0, L)).  No reference
 * counterpart. */
DEM_API int dem_overlap_pairs(dem_ctx *ctx, int n, const double *x, const double *y, const double *z,
                              const double *r, double L, int periodic, int table_size, int32_t *pairs,
                              int64_t pair_capacity, int64_t *counts, void *stream);

/* Allocation-free spatial-hash detection.  This entry point has no
 * counterpart in the reference: it is for callers that cannot call
 * cudaMalloc when they detect collisions (a fixed device-memory budget handed
 * over up front, a control loop that must not take cudaMalloc's device-wide
 * synchronisation between steps, or an allocator owned by another
 * component).  Same arguments and pair output as dem_hash_detect, without a
 * context: the workspace is a fixed device array inside the library (about
 * 2.9 MB, held on every GPU that loads the library until the process exits).
 * Overflow: with no context there is no error flag to read, so a caller sees
 * a short pair buffer only as counts[0] > pair_capacity (the buffer then holds
 * the lexicographically first pair_capacity pairs).  Limits: n <= 65536 droplets and table_size <= 131072
 * buckets; larger sizes return DEM_E_CAPACITY; bad pointers DEM_E_INVALID;
 * CUDA failures DEM_E_CUDA (no message: there is no context).  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.  All
 * calls share the one array: calls that overlap on the GPU (different streams
 * or host threads at the same time) race and corrupt each other's results. */
DEM_API int dem_hash_detect_noalloc(int n, const double *x, const double *y, const double *z, const double *r,
                                    double L, int periodic, int table_size, int32_t *pairs, int64_t pair_capacity,
                                    int64_t *counts, void *stream);

/* Collision counts between volume classes from detected pairs (dem_hash_detect
 * output: pairs, counts[0]): matrix[b_i][b_j] += 1 and matrix[b_j][b_i] += 1 for
 * each of the first min(counts[0], pair_capacity) pairs.  bins: device
 * int32[n]; matrix: device uint32[nbins^2], zeroed here.
 * Replaces DirectCollisionFrequency.compute, pbm/collision_frequency/direct_collision_freq.py:17-41. */
DEM_API int dem_pair_bin_matrix(dem_ctx *ctx, const int32_t *pairs, const int64_t *num_pairs, int64_t pair_capacity,
                                const int32_t *bins, int nbins, uint32_t *matrix, void *stream);

/* ---- droplet generator ------------------------------------------------ */
/* Seeded droplets with overlap rejection, written to DEVICE x, y, z, r:
 * radii uniform in [rmin, rmax], positions uniform in [lo, hi)^3; then, round
 * by round, the droplets just drawn that overlap any droplet (distance <=
 * r_i + r_j + minimum_distance; minimum image when periodic, with period
 * hi - lo) are drawn again, until none is left.  More than max_rounds rounds:
 * DEM_E_INVALID (the reference raises ValueError after 1,000).  Random numbers
 * are a counter-based SplitMix64 stream of (seed, purpose, round, droplet).
 * *rounds_out (host, may be NULL): rounds used.  Synchronises `stream`.
 * Replaces UniformDropletGenerator.generate / reseed_overlaping_droplets,
 * dem/particle_generator/uniform_droplet_generator.py:45-164 (whose overlap
 * test is the plain distance: periodic = 0). */
DEM_API int dem_generate_droplets(dem_ctx *ctx, int n, unsigned long long seed, double lo, double hi, double rmin,
                                  double rmax, double minimum_distance, int periodic, int max_rounds, double *x,
                                  double *y, double *z, double *r, int *rounds_out, void *stream);

/* ---- coalescence ------------------------------------------------------ */
/* Greedy merge of the colliding pairs in (i, j) order; survivors keep their
 * order and the merged droplets are appended in pair order.
 *   r_new = (r_a^3 + r_b^3)^(1/3),  x_new = (x_a r_a^3 + x_b r_b^3) / (r_a^3 + r_b^3)  (no MIC)
 * num_pairs: device int64 (counts[0] of dem_hash_detect).  Outputs must not
 * alias inputs.  n_out: device int32, the new droplet count.  merged: optional
 * device int32[n][2] receiving the merged (a, b) pairs in merge order.
 * Replaces DropletSolution.generate_next_solution,
 * dem/solution/droplet_solution.py:208-287. */
DEM_API int dem_merge(dem_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *r,
              const int32_t *pairs, const int64_t *num_pairs, double *xo, double *yo, double *zo, double *ro,
              int32_t *n_out, int32_t *merged, void *stream);

/* ---- flat Barnes-Hut octree (reference drop-in, FP64) ------------------ */
/* Same tree, node numbering, aggregates and walks as FlatOctree
 * (dem/octree/flat_tree.py:36-1630): bit-identical forces and velocities. */
typedef struct dem_tree dem_tree;

/* Node pool of max_nodes nodes (the reference sizes it max(4 N / mpl, 1024),
 * flat_tree.py:63-66) and room for `capacity` particles. */
DEM_API int dem_tree_create(dem_ctx *ctx, int capacity, int max_nodes, dem_tree **out);
DEM_API void dem_tree_destroy(dem_tree *tree);

/* FlatOctree.build, flat_tree.py:180-246: level-by-level subdivision of
 * leaves holding more than mpl droplets (skipped once the pool is full),
 * leaf slots, next pointers, R^3 aggregates.  Synchronises `stream` once
 * per level.  DEM_E_CAPACITY when n > capacity (the reference's ValueError,
 * :184-189). */
DEM_API int dem_tree_build(dem_tree *tree, int n, const double *x, const double *y, const double *z,
                           const double *r, double L, int periodic, int mpl, void *stream);

/* _compute_forces_kernel, flat_tree.py:783-894 (MAC s^2 < theta_sq D^2).
 * The forces are also kept for the velocity walk. */
DEM_API int dem_tree_forces(dem_tree *tree, double m_const, double theta_sq, double *fx, double *fy, double *fz,
                            void *stream);

/* Force sums and raw moments bottom-up, flat_tree.py:556-777.  fx == NULL
 * uses the forces kept by dem_tree_forces (_propagate_forces_from_fields). */
DEM_API int dem_tree_propagate_forces(dem_tree *tree, const double *fx, const double *fy, const double *fz,
                                      void *stream);

/* Stokeslet walk (stokes_factor <= 0, flat_tree.py:1000-1280) or total
 * velocity walk (stokes_factor > 0, :1326-1588), correction off.  fx..fz are
 * the leaf forces (forces_np); NULL uses the kept forces. */
DEM_API int dem_tree_velocity(dem_tree *tree, const double *fx, const double *fy, const double *fz, double eta_const,
                              double theta_sq, double stokes_factor, double *vx, double *vy, double *vz,
                              void *stream);

/* Attaches a periodic-image correction (dem_corr_create) to the velocity
 * walks, NULL detaches it.  Then the Stokeslet walk adds each leaf pair's and
 * each accepted node's correction term right after its Stokeslet term and
 * the self term self_coeff * F_i after the walk; the total-velocity walk
 * adds the pair and node terms only, as the reference does
 * (flat_tree.py:1070-1131, :1171-1213, :1271-1276; bit-identical).  The grid
 * must outlive its use by the tree.
 * Replaces FlatOctree.load_periodic_correction, flat_tree.py:141-167. */
DEM_API int dem_tree_set_correction(dem_tree *tree, const dem_corr *corr);

/* Collision counts between volume classes over the built tree: every pair
 * j > i with |MIC(x_j - x_i)|^2 <= (r_i + r_j)^2 adds 1 to matrix[b_i][b_j] and
 * to matrix[b_j][b_i]; nodes are pruned when the squared distance to their box
 * exceeds (r_i + max radius in the node)^2, with the reference's periodic box
 * distance (per axis: gap > L/2 -> L - gap).  bins: device int32[n] class of
 * each droplet (caller order), 0 <= b < nbins; matrix: device uint32[nbins^2],
 * zeroed here.
 * Replaces TreeCollisionFrequency.compute, pbm/collision_frequency/tree_collision_freq.py:43-175. */
DEM_API int dem_tree_collision_matrix(dem_tree *tree, const int32_t *bins, int nbins, uint32_t *matrix, void *stream);

/* Host int64[8]: node_count, parent_count, leaf_slot_count, max_nodes,
 * levels, num_particles, pool_exhausted, capacity. */
DEM_API int dem_tree_stats(const dem_tree *tree, int64_t *out);

/* Copies node data into DEVICE buffers of node_count entries (NULL skips):
 * count, first_child, next, leaf_start (int32); r3 (4 per node: R3 sum and
 * R3-weighted coordinate sums); fs (12 per node: force sum, 9 moments). */
DEM_API int dem_tree_nodes(dem_tree *tree, int32_t *count, int32_t *first_child, int32_t *next, int32_t *leaf_start,
                           double *r3, double *fs, void *stream);
DEM_API int dem_tree_leaf_indices(dem_tree *tree, int32_t *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DEM_B200_H */
