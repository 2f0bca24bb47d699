/*
 * ocu_b200.h -- C ABI of the B200-native OpenCurrent projection-step library
 * (libocu_b200.so).  Plain pointers, sizes and opaque handles; no C++ or torch types.
 *
 * Conventions shared by every entry point:
 *   - Return an ocu_status; OCU_OK == 0.  ocu_last_error() gives a human-readable message for
 *     the calling thread's most recent failure.  This replaces the reference's bool returns +
 *     sticky ErrorHandler flag (ocuequation/error_handler.h:27-57); the C++ facade in
 *     include/ocu/ maps it back to bool + any_error().
 *   - Every device operation is enqueued on a caller-chosen CUDA stream (ocu_stream is
 *     layout-compatible with cudaStream_t; NULL = legacy default stream).  The reference uses
 *     ThreadManager::get_compute_stream() (ocuutil/thread.h:86-87).  Nothing here calls
 *     cudaDeviceSynchronize; an entry point only blocks when it must hand a number back to the
 *     host (norms, time steps) and says so.
 *   - Grids follow the Grid3DDevice<T> layout contract of ocu_types.h; kernels are built for
 *     sm_100a only and there is no CPU fallback: on a machine without a B200 every compute
 *     entry point returns OCU_ERR_CUDA.
 */
#ifndef OCU_B200_H
#define OCU_B200_H

#include "ocu_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *ocu_stream; /* == cudaStream_t */

typedef enum ocu_status {
  OCU_OK = 0,
  OCU_ERR_INVALID_VALUE = 1,  /* bad argument (NaN h, negative tolerance, bad BC type ...) */
  OCU_ERR_LAYOUT = 2,         /* grid dimensions or padded layouts do not match */
  OCU_ERR_CUDA = 3,           /* a CUDA runtime call or kernel launch failed */
  OCU_ERR_NOT_CONVERGED = 4,  /* solver stopped at max_iter above tolerance */
  OCU_ERR_NOT_INITIALIZED = 5,
  OCU_ERR_ALLOC = 6,
  OCU_ERR_UNSUPPORTED = 7,
  OCU_ERR_TIMEOUT = 8         /* a bounded device-side wait gave up (status word set) */
} ocu_status;

typedef struct ocu_grid ocu_grid;
typedef struct ocu_mg ocu_mg;
typedef struct ocu_project ocu_project;
typedef struct ocu_ns ocu_ns;

/* ---- library ------------------------------------------------------------------------- */
const char *ocu_last_error(void);
/* Version string and the compute capability the kernels were built for ("sm_100a"). */
const char *ocu_version(void);
/* Number of kernel launches this library issued on the calling process (all streams). */
unsigned long long ocu_kernel_launch_count(void);

/* ---- grids: Grid3DDevice<T> (ocustorage/grid3d.h:219-264, grid3ddev.cu) ---------------- */
/* Layout rule of Grid3DDevice<T>::init (grid3ddev.cu:358-400); host-only. */
ocu_status ocu_layout_compute(int nx, int ny, int nz, int gx, int gy, int gz, int padx,
                              int pady, int padz, ocu_layout *out);
/* Grid3DDevice<T>::init: cudaMalloc + zero fill. */
ocu_status ocu_grid_create(ocu_dtype dtype, int nx, int ny, int nz, int gx, int gy, int gz,
                           int padx, int pady, int padz, ocu_grid **out);
/* Borrow caller device memory of layout->allocated elements (e.g. a torch tensor). */
ocu_status ocu_grid_wrap(ocu_dtype dtype, const ocu_layout *layout, void *device_buffer,
                         ocu_grid **out);
void ocu_grid_destroy(ocu_grid *g);
ocu_status ocu_grid_info(const ocu_grid *g, ocu_layout *layout, ocu_dtype *dtype,
                         void **device_buffer);
/* copy_all_data host<->device (grid3ddev.cu:244-258; grid3dhost.cu): the whole padded
 * buffer, synchronous with respect to the stream (the call returns after the copy). */
ocu_status ocu_grid_upload(ocu_grid *g, const void *host_buffer, ocu_stream s);
ocu_status ocu_grid_download(const ocu_grid *g, void *host_buffer, ocu_stream s);
/* Same, asynchronous: host_buffer should be pinned and must stay valid until the stream
 * reaches the copy. */
ocu_status ocu_grid_upload_async(ocu_grid *g, const void *host_buffer, ocu_stream s);
ocu_status ocu_grid_download_async(const ocu_grid *g, void *host_buffer, ocu_stream s);
/* Grid3DDevice<T>::copy_all_data<S> (grid3ddev.cu:260-279): element-wise, converting. */
ocu_status ocu_grid_copy_all_data(ocu_grid *dst, const ocu_grid *src, ocu_stream s);
/* clear_zero / clear(T) (grid3ddev.cu:221-242). */
ocu_status ocu_grid_clear(ocu_grid *g, double value, ocu_stream s);
/* linear_combination (grid3ddev.cu:283-349): g2 == NULL gives this = alpha1*g1. */
ocu_status ocu_grid_linear_combination(ocu_grid *result, double alpha1, const ocu_grid *g1,
                                       double alpha2, const ocu_grid *g2, ocu_stream s);
/* reduce_* (grid3dops.cu:26-130): same fold order as the reference; blocks the host. */
ocu_status ocu_grid_reduce(const ocu_grid *g, ocu_reduce_op op, double *result, ocu_stream s);

/* Largest number of 256-row blocks ocu_grid_reduce_noalloc can fold: grids with
 * nx*ny <= 256 * OCU_REDUCE_NOALLOC_MAX_BLOCKS (1,048,576 rows, e.g. 1024 x 1024 planes). */
#define OCU_REDUCE_NOALLOC_MAX_BLOCKS 4096
/* ocu_grid_reduce without any device allocation.  (No counterpart in the reference: it exists
 * for callers that must not allocate device memory when they ask for a norm -- a host whose
 * allocator already owns the whole device, a plugin host that reserves all memory up front and
 * forbids later allocations, or a latency-critical loop that must stay off the allocator.)
 * Same result as ocu_grid_reduce, bit for bit.  Its scratch is one static array in the
 * library's device image (about 33 KB, held on every GPU that loads the library until the
 * process exits); larger grids than the limit above are rejected with OCU_ERR_INVALID_VALUE.
 * All calls on a device share that array and it keeps the previous call's contents (each call
 * clears what must start at zero), so calls that overlap on the GPU -- other streams or host
 * threads without ordering between them -- race and must be serialised by the caller.  The
 * first call on a device looks up the array's device address while that device is current and
 * keeps it for the life of the process, so the device must not be reset (cudaDeviceReset)
 * after that first call.  Every call blocks the host until the result is back, so the
 * function cannot be called on a stream that is being captured into a graph. */
ocu_status ocu_grid_reduce_noalloc(const ocu_grid *g, ocu_reduce_op op, double *result, ocu_stream s);

/* ---- ghost cells (ocustorage/grid3dboundary.h:26-70) --------------------------------- */
/* apply_3d_boundary_conditions_level1 (variant OCU_BC_LEVEL1, one launch instead of three)
 * and ..._level1_nocorners (OCU_BC_LEVEL1_NOCORNERS). */
ocu_status ocu_apply_boundary_conditions(ocu_grid *g, const ocu_bc_set *bc, double hx,
                                         double hy, double hz, ocu_bc_variant variant,
                                         ocu_stream s);
/* apply_3d_mac_boundary_conditions_level1 (grid3dboundary.cu:823-900). */
ocu_status ocu_apply_mac_boundary_conditions(ocu_grid *u, ocu_grid *v, ocu_grid *w,
                                             const ocu_bc_set *bc, double hx, double hy,
                                             double hz, ocu_stream s);

/* ---- stateless stencils ---------------------------------------------------------------- */
/* Sol_Divergence3DDevice<T>::solve (sol_divergence3ddev.cu:23-88). */
ocu_status ocu_divergence(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w,
                          ocu_grid *divergence, int nx, int ny, int nz, double hx, double hy,
                          double hz, ocu_stream s);
/* Sol_Gradient3DDevice<T>::solve: u += coefficient * grad(phi) (sol_gradient3ddev.cu:24-88). */
ocu_status ocu_gradient_add(ocu_grid *u, ocu_grid *v, ocu_grid *w, const ocu_grid *phi,
                            double coefficient, double hx, double hy, double hz, ocu_stream s);
/* Sol_SelfAdvection3DDevice<T>::solve (sol_selfadvection3ddev.cu:584-590, kernels :135-337). */
ocu_status ocu_advect_self(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w,
                           ocu_grid *dudt, ocu_grid *dvdt, ocu_grid *dwdt, int nx, int ny,
                           int nz, double hx, double hy, double hz, ocu_interpolation interp,
                           ocu_stream s);
/* Sol_PassiveAdvection3DDevice<T>::solve (sol_passiveadvection3ddev.cu:31-136). */
ocu_status ocu_advect_passive(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w,
                              const ocu_grid *phi, ocu_grid *dphidt, int nx, int ny, int nz,
                              double hx, double hy, double hz, ocu_interpolation interp,
                              ocu_stream s);
/* Sol_LaplacianCentered3DDevice<T>::solve: dphidt += coefficient * lap(phi) over
 * (nx,ny,nz) cells (sol_laplaciancent3ddev.cu:28-109). */
ocu_status ocu_laplacian_add(const ocu_grid *phi, ocu_grid *dphidt, int nx, int ny, int nz,
                             double hx, double hy, double hz, double coefficient,
                             ocu_stream s);

/* ---- multigrid pressure solver (Sol_MultigridPressure3DDevice<T>,
 *      ocuequation/sol_mgpressure3d.h:36-248) ------------------------------------------- */
typedef enum ocu_mg_kind {
  OCU_MG_F32 = 0,              /* Sol_MultigridPressure3DDeviceF */
  OCU_MG_F64 = 1,              /* Sol_MultigridPressure3DDeviceD */
  OCU_MG_MIXED_IR = 2,         /* FP32 V-cycles inside FP64 iterative refinement (new) */
  OCU_MG_MIXED_WARMSTART = 3   /* reference Sol_MultigridPressureMixed3DDeviceD algorithm
                                  (sol_mgpressuremixed3ddevd.cpp:79-100) */
} ocu_mg_kind;

/* Public fields of Sol_MultigridPressure3DBase / ...Device (sol_mgpressure3d.h:86-90, 163). */
typedef struct ocu_mg_params {
  ocu_bc_set bc;
  int nu1, nu2;
  int convergence;               /* ocu_convergence */
  int make_symmetric_operator;
  int disable_relax_on_host;     /* kept for API parity: the coarsest level is always relaxed
                                    on the device here; 0 = one CTA runs the reference host
                                    routine's arithmetic and ghost fills, 1 = the device
                                    colour-sweep kernels relax it */
  int ir_inner_cycles;           /* OCU_MG_MIXED_IR only: FP32 fine-level cycles per
                                    correction (0 = default 4) */
  int store_residual_grids;      /* 1 = keep r_grid(level) filled (read_r); costs N*s */
  int unfused;                   /* 1 = one launch per reference operation (no fused ghost
                                    writes, no fused residual+restriction, no tail kernel);
                                    same results, for A/B timing */
  int tail_cells;                /* levels with at most this many cells run in one single-CTA
                                    kernel per cycle; 0 = default (64), < 0 = off */
  int sweep_cells;               /* levels with at least this many cells relax both colours in
                                    one TMA-fed pass (out of place, same results; Dirichlet and
                                    Neumann faces only); <= 0 = off (the default) */
  int ir_inner_exact;            /* OCU_MG_MIXED_IR only: 0 (default) = the FP32 correction
                                    solves run on red/black split colour arrays with fused
                                    multiply-adds (this library's own inner solver, checked
                                    against FP64 multigrid at the tolerance); 1 = they run on
                                    the reference-layout kernels, bit-identical to the CPU
                                    oracle's restatement.  Hierarchies the split solver does not
                                    take (one level, an odd periodic axis, a coarsest level
                                    larger than 48 KB of shared memory) always use the latter. */
  int wait_limit;                /* polls of a bounded device wait (the two-colour TMA pass
                                    waiting for its loads) before it gives up; the solve then
                                    returns OCU_ERR_TIMEOUT and the next one starts clean.
                                    0 = the default (about a second).  Negative: a test of that
                                    path -- each launch of the pass first waits -wait_limit polls
                                    on a barrier nothing completes, gives up before issuing any
                                    load, and the solve reports OCU_ERR_TIMEOUT */
} ocu_mg_params;

typedef struct ocu_mg_stats {
  int num_levels;
  int vcycles;                   /* fine-level cycles of the last do_fmg / IR inner total */
  int outer_iterations;          /* OCU_MG_MIXED_IR: refinement steps of the last solve */
  double last_l2, last_linf;     /* norms of the last convergence check */
  double omega;
} ocu_mg_stats;

/* Fills the reference constructor defaults (sol_mgpressure3d.cpp:26-40). */
void ocu_mg_params_default(ocu_mg_params *p);
ocu_status ocu_mg_create(ocu_mg_kind kind, const ocu_mg_params *params, ocu_mg **out);
void ocu_mg_destroy(ocu_mg *mg);
ocu_status ocu_mg_set_params(ocu_mg *mg, const ocu_mg_params *params);
ocu_status ocu_mg_get_params(const ocu_mg *mg, ocu_mg_params *params);
ocu_status ocu_mg_set_stream(ocu_mg *mg, ocu_stream s);
/* initialize_storage (sol_mgpressure3ddev.cu:376-482).  rhs is borrowed, not copied; its dtype
 * must be F32 for OCU_MG_F32 and F64 otherwise; ghost >= 1. */
ocu_status ocu_mg_initialize_storage(ocu_mg *mg, int nx, int ny, int nz, double hx, double hy,
                                     double hz, ocu_grid *rhs);
/* solve(residual, tol, max_iter) (sol_mgpressure3d.cpp:332-370): OCU_OK when converged,
 * OCU_ERR_NOT_CONVERGED otherwise (residual still written).  Blocks the host. */
ocu_status ocu_mg_solve(ocu_mg *mg, double *residual, double tolerance, int max_iter);
ocu_status ocu_mg_run_vcycles(ocu_mg *mg, int count);   /* sol_mgpressure3d.cpp:372-384 */
ocu_status ocu_mg_run_fmg(ocu_mg *mg, int count);       /* sol_mgpressure3d.cpp:386-398 */
/* pressure() and read_u/r/b(level) (sol_mgpressure3d.h:173-179); which = 'u','r','b'.
 * The handle is owned by the solver. */
ocu_grid *ocu_mg_pressure(ocu_mg *mg);
ocu_grid *ocu_mg_level_grid(ocu_mg *mg, char which, int level);
ocu_status ocu_mg_get_stats(const ocu_mg *mg, ocu_mg_stats *stats);
/* The level operations the cycle is built from (protected in the reference,
 * sol_mgpressure3d.h:76-80), exposed for testing and kernel timing.  core = 0 acts on the
 * interface precision, core = 1 on the FP32 hierarchy of a mixed solver, core = 2 on the
 * red/black split FP32 hierarchy of an OCU_MG_MIXED_IR solver (relax order 0 or 1; restriction
 * into the next level without norms).  They enqueue work and
 * return without waiting, except restrict_residuals when a norm is requested. */
/* relax(level, iterations, order): order 0 red-black, 1 black-red, 2 symmetric
 * (sol_mgpressure3ddev.cu:190-248). */
ocu_status ocu_mg_relax(ocu_mg *mg, int core, int level, int iterations, int order);
/* One colour-sweep launch, no ghost refresh (sol_mgpressure3ddevf.cu:200-252). */
ocu_status ocu_mg_relax_sweep(ocu_mg *mg, int core, int level, int color);
/* restrict_residuals(fine, coarse, l2, linf) (sol_mgpressure3ddev.cu:250-279); NULL skips a norm. */
ocu_status ocu_mg_restrict_residuals(ocu_mg *mg, int core, int fine, int coarse, double *l2,
                                     double *linf);
/* prolong(coarse, fine) + ghost refresh (sol_mgpressure3ddev.cu:284-297). */
ocu_status ocu_mg_prolong(ocu_mg *mg, int core, int coarse, int fine);
/* Wait for all work the solver enqueued. */
ocu_status ocu_mg_synchronize(ocu_mg *mg);

/* ---- multi-image multigrid (Sol_MultigridPressure3DDeviceCo<T>) ---------------------------
 * sol_mgpressure3d.h:184-242, sol_mgpressure3dco.cu:39-529.  The domain is split along x into
 * `num_images` slabs of nx_local x ny x nz, one per image; an image lives on a device (several
 * images may share one).  The reference runs one host thread per image with host-staged
 * barrier exchanges (coarray.h:50-113); here one host thread drives every image in lockstep:
 * each image has its own stream, the one-plane x halo is copied device to device into the
 * receiving image's ghost plane (peer access over NVLink across devices) after every ghost
 * refresh, ordered by events, so no kernel waits on another.  Levels whose global cell count
 * is at most the cutoff (grid_size_for_cutoff, 64^3 by default) are gathered onto image 0 and
 * scattered back before the prolongation, as in the reference.  Norms are each image's
 * reduction folded in image order on the host.  The handle is an ocu_mg of kind OCU_MG_F32 or
 * OCU_MG_F64: ocu_mg_solve / run_vcycles / run_fmg / set_params / get_stats / set_stream (image
 * 0's stream, on devices[0]) / synchronize / destroy apply, and core 0 of the level operations
 * acts on all images. */
typedef struct ocu_mgco_plan {
  int num_levels;     /* levels of the global hierarchy */
  int cutoff_level;   /* first level held whole by image 0 (num_levels: none) */
  int neg_image;      /* image across the x- face, -1 at the domain's face */
  int pos_image;      /* image across the x+ face, -1 at the domain's face */
  ocu_bc_set local_bc;  /* this image's faces at level 0: BC_NONE where a neighbour's plane lands */
} ocu_mgco_plan;
/* Host-only: the decomposition of one image (sol_mgpressure3dco.cu:242-300, 420-435). */
ocu_status ocu_mgco_plan_compute(int nx_local, int ny, int nz, int num_images, int image,
                                 long long cutoff_cells, const ocu_bc_set *bc, ocu_mgco_plan *out);
/* kind: OCU_MG_F32 or OCU_MG_F64.  devices: num_images device ordinals (NULL: all 0). */
ocu_status ocu_mgco_create(ocu_mg_kind kind, const ocu_mg_params *params, int num_images,
                           const int *devices, ocu_mg **out);
/* grid_size_for_cutoff (sol_mgpressure3dco.cu:223); before initialize_storage. */
ocu_status ocu_mgco_set_cutoff_cells(ocu_mg *mg, long long cells);
/* initialize_storage (sol_mgpressure3dco.cu:240-520): rhs[i] is image i's slab (borrowed),
 * all with the same layout, ghost >= 1.  The global grid is (nx_local * num_images) x ny x nz;
 * every level above the cutoff must split evenly across the images. */
ocu_status ocu_mgco_initialize_storage(ocu_mg *mg, int nx_local, int ny, int nz, double hx,
                                       double hy, double hz, ocu_grid *const *rhs);
/* co_pressure() of an image (its slab of u at level 0); owned by the solver. */
ocu_grid *ocu_mgco_pressure(ocu_mg *mg, int image);
int ocu_mgco_num_images(const ocu_mg *mg);
int ocu_mgco_cutoff_level(const ocu_mg *mg);

/* ---- differentiable advection + projection (periodic MAC grid) ----------------------------
 * No single counterpart in the reference: the transposes of Sol_SelfAdvection3DDevice /
 * Sol_PassiveAdvection3DDevice (sol_selfadvection3ddev.cu:135-337,
 * sol_passiveadvection3ddev.cu:31-78) with the upwind choice frozen, and a chain of `steps`
 * forward-Euler steps (passive + self advection, then projection) with checkpoints every
 * `checkpoint_every` steps.  Cotangents use the plain sum inner product over the nx*ny*nz
 * cells/faces; ghost and padding entries of returned cotangents are zero. */
/* lam_phi = lam_dphi + c (d dphi/d phi)^T lam_dphi;  lam_{u,v,w} += c (d dphi/d {u,v,w})^T lam_dphi */
ocu_status ocu_advect_passive_adjoint(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w,
                                      const ocu_grid *phi, const ocu_grid *lam_dphi, ocu_grid *lam_phi,
                                      ocu_grid *lam_u, ocu_grid *lam_v, ocu_grid *lam_w, int nx, int ny,
                                      int nz, double c, double hx, double hy, double hz, int interp,
                                      ocu_stream s);
/* lam_{u,v,w} += c (d (du,dv,dw) / d (u,v,w))^T (lam_du, lam_dv, lam_dw) */
ocu_status ocu_advect_self_adjoint(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w,
                                   const ocu_grid *lam_du, const ocu_grid *lam_dv,
                                   const ocu_grid *lam_dw, ocu_grid *lam_u, ocu_grid *lam_v,
                                   ocu_grid *lam_w, int nx, int ny, int nz, double c, double hx,
                                   double hy, double hz, int interp, ocu_stream s);
typedef struct ocu_adj ocu_adj;
ocu_status ocu_adj_create(ocu_dtype dtype, int nx, int ny, int nz, double hx, double hy, double hz,
                          int steps, int checkpoint_every, double dt, int interp, double proj_tol,
                          ocu_adj **out);
void ocu_adj_destroy(ocu_adj *a);
ocu_status ocu_adj_set_stream(ocu_adj *a, ocu_stream s);
/* layouts of the chain's grids: 'u', 'v', 'w' (MAC faces) and 't' (the scalar) */
ocu_status ocu_adj_layout(const ocu_adj *a, char which, ocu_layout *layout);
/* runs the chain from (u0, v0, w0, phi0), keeps the checkpoints, writes the final scalar */
ocu_status ocu_adj_forward(ocu_adj *a, const ocu_grid *u0, const ocu_grid *v0, const ocu_grid *w0,
                           const ocu_grid *phi0, ocu_grid *phi_out);
/* given the cotangent of the final scalar, the cotangents of the initial velocity and scalar
 * of the last forward run (segments recomputed from the checkpoints) */
ocu_status ocu_adj_backward(ocu_adj *a, const ocu_grid *lam_phi, ocu_grid *lam_u0, ocu_grid *lam_v0,
                            ocu_grid *lam_w0, ocu_grid *lam_phi0);

/* ---- ensembles of independent pressure solves ---------------------------------------------
 * No single counterpart in the reference: many Sol_MultigridPressure3DDevice<T>::solve calls
 * (sol_mgpressure3d.cpp:332-370) on right-hand sides of uneven sizes, run together.  Members
 * with equal dimensions and spacings form a size class; every multigrid step of a class is one
 * launch over all its members, convergence is decided per member on the device, and each class
 * replays one CUDA graph per V-cycle.  Each member's pressure is bit-identical to a single
 * solver's with the same parameters (convergence must be OCU_CONVERGENCE_L2; every face BC must
 * allow fused ghost writes: no BC_NONE, even periodic axes). */
typedef struct ocu_ens ocu_ens;
typedef struct ocu_ens_tuning {
  int nu1, nu2;          /* smoothing counts of the class's V-cycles */
  int relax_block[3];    /* colour-sweep CTA shape: k pairs, j, i (product <= 256) */
  double ms;             /* autotuner: measured solve time of the class with this setting */
} ocu_ens_tuning;
/* dims: 3 ints per member (nx, ny, nz); h: 3 doubles per member (hx, hy, hz); params as for
 * ocu_mg_create (bc, nu1, nu2, make_symmetric_operator, disable_relax_on_host are used). */
ocu_status ocu_ens_create(ocu_dtype dtype, int members, const int *dims, const double *h,
                          const ocu_mg_params *params, ocu_ens **out);
void ocu_ens_destroy(ocu_ens *e);
/* Solves start after prior work on this stream; ocu_ens_solve returns when all is done. */
ocu_status ocu_ens_set_stream(ocu_ens *e, ocu_stream s);
/* Views of one member's right-hand side and pressure (standard layout of its dimensions,
 * ghost 1); owned by the ensemble, valid until ocu_ens_destroy, never ocu_grid_destroy'ed. */
ocu_status ocu_ens_rhs(ocu_ens *e, int member, ocu_grid **out);
ocu_status ocu_ens_pressure(ocu_ens *e, int member, ocu_grid **out);
/* tol: one absolute L2 tolerance per member; each member runs the FMG + V-cycle schedule of
 * solve() from its current pressure, at most max_iter + 1 level-0 cycles.  *converged gets the
 * number of members that reached their tolerance; OCU_ERR_NOT_CONVERGED if some did not. */
ocu_status ocu_ens_solve(ocu_ens *e, const double *tol, int max_iter, int *converged);
/* vcycles and last_l2 of the member's last solve. */
ocu_status ocu_ens_member_stats(const ocu_ens *e, int member, ocu_mg_stats *stats);
ocu_status ocu_ens_num_classes(const ocu_ens *e, int *n);
ocu_status ocu_ens_class_info(const ocu_ens *e, int cls, int *dims, int *members,
                              ocu_ens_tuning *tuning);
ocu_status ocu_ens_set_tuning(ocu_ens *e, int cls, const ocu_ens_tuning *tuning);
/* Per class, times whole solves from a zero guess for several smoothing pairs and colour-sweep
 * shapes and keeps the fastest that converges every member; leaves every pressure zeroed. */
ocu_status ocu_ens_autotune(ocu_ens *e, const double *tol, int max_iter);

/* ---- preconditioned conjugate gradients (Sol_PCGPressure3DDevice<T>, sol_pcgpressure3d.h:41-97) --
 * Solves L p = rhs, L = -div(c grad) with a cell coefficient grid c (the variable-coefficient
 * pressure equation), by CG with no preconditioner, Jacobi, multigrid (FMG or V-cycles of the
 * constant-coefficient multigrid solver on the residual, sign flipped) or BFBT (multigrid then
 * Jacobi), restarting the residual from rhs - L p every 25 iterations, as the reference does
 * (sol_pcgpressure3d.cu:335-457).  Faces must be periodic or Neumann.  solve() returns
 * OCU_ERR_NOT_CONVERGED (the reference's false) when sqrt(<r, M^-1 r>) stays at or above the
 * tolerance after max_iter + 1 iterations; *residual is that norm (OCU_CONVERGENCE_L2) or
 * max |r|.  Bit-identical to the CPU oracle's restatement. */
typedef struct ocu_pcg ocu_pcg;
typedef struct ocu_pcg_params {
  ocu_bc_set bc;
  int convergence;        /* OCU_CONVERGENCE_L2 (default) or OCU_CONVERGENCE_LINF */
  int preconditioner;     /* ocu_precond; default OCU_PRECOND_BFBT */
  int multigrid_cycles;   /* default 2 */
  int multigrid_use_fmg;  /* default 1; 0 = V-cycles */
} ocu_pcg_params;
/* The reference constructor's defaults (sol_pcgpressure3d.cu:160-171), faces Neumann. */
void ocu_pcg_params_default(ocu_pcg_params *p);
ocu_status ocu_pcg_create(ocu_dtype dtype, const ocu_pcg_params *params, ocu_pcg **out);
void ocu_pcg_destroy(ocu_pcg *s);
ocu_status ocu_pcg_set_stream(ocu_pcg *s, ocu_stream stream);
/* convergence, preconditioner and the multigrid counts take effect at the next solve; bc only
 * before initialize_storage */
ocu_status ocu_pcg_set_params(ocu_pcg *s, const ocu_pcg_params *params);
/* initialize_storage(nx, ny, nz, hx, hy, hz, rhs, coefficient) (sol_pcgpressure3d.cu:604-654):
 * spacings are float, as in the reference; rhs and coefficient share one layout (ghost >= 1) and
 * are borrowed (the coefficient's face ghosts are written at each solve); the pressure is
 * allocated congruent and cleared. */
ocu_status ocu_pcg_initialize_storage(ocu_pcg *s, int nx, int ny, int nz, float hx, float hy, float hz,
                                      ocu_grid *rhs, ocu_grid *coefficient);
ocu_status ocu_pcg_solve(ocu_pcg *s, double *residual, double tolerance, int max_iter);
ocu_status ocu_pcg_pressure(ocu_pcg *s, ocu_grid **out);
/* CG iterations of the last solve */
ocu_status ocu_pcg_iterations(const ocu_pcg *s, int *out);

/* ---- grid files (NetCDFGrid3DWriter / NetCDFGrid3DReader, gridnetcdf.h:67-183) -------------
 * The reference's NetCDF grid files, written and read without libnetcdf in the NetCDF classic
 * format (CDF-1, or CDF-2 when the data passes 2 GB): an unlimited "Time" dimension and float
 * "Time" variable, global attributes nx, ny, nz, hx, hy, hz, one coordinate dimension + float
 * variable per axis offset (XAxisCentered, XAxisUFace, XAxisOffset%.4f, ...), and each grid
 * variable on (Time, X, Y, Z).  Data are host grids: the interior origin, the x and y strides
 * in elements (z contiguous) and the interior extents, of the variable's type.  The writer keeps
 * the data in memory and writes the file at close. */
typedef struct ocu_nc_writer ocu_nc_writer;
typedef struct ocu_nc_reader ocu_nc_reader;
/* open (gridnetcdf.cpp: nc_create with NC_CLOBBER): creates / truncates the file now */
ocu_status ocu_nc_writer_open(const char *path, int nx, int ny, int nz, float hx, float hy, float hz,
                              ocu_nc_writer **out);
/* define_variable(name, nc_type, staggering, offsets used for OCU_GS_CUSTOM) */
ocu_status ocu_nc_writer_define_variable(ocu_nc_writer *w, const char *name, int nc_type, int staggering,
                                         float offsetx, float offsety, float offsetz);
ocu_status ocu_nc_writer_add_time_level(ocu_nc_writer *w, float time, int *level);
/* add_data: level 0 of a file without time levels adds time 0 first, as the reference does */
ocu_status ocu_nc_writer_add_data(ocu_nc_writer *w, const char *name, const void *origin, int nc_type,
                                  long long xstride, long long ystride, int nx, int ny, int nz, int time_level);
/* the same from a device grid (downloaded first) */
ocu_status ocu_nc_writer_add_grid(ocu_nc_writer *w, const char *name, const ocu_grid *g, int time_level);
/* writes the file and frees the writer */
ocu_status ocu_nc_writer_close(ocu_nc_writer *w);
ocu_status ocu_nc_reader_open(const char *path, ocu_nc_reader **out);
void ocu_nc_reader_close(ocu_nc_reader *r);
ocu_status ocu_nc_reader_info(const ocu_nc_reader *r, int *nx, int *ny, int *nz, float *hx, float *hy, float *hz,
                              int *num_time_levels);
ocu_status ocu_nc_reader_get_time(const ocu_nc_reader *r, int time_level, float *time);
/* list_variables / variable_type / variable_size: the grid variables in file order */
ocu_status ocu_nc_reader_num_variables(const ocu_nc_reader *r, int *n);
ocu_status ocu_nc_reader_variable(const ocu_nc_reader *r, int index, char *name, int name_size, int *nc_type,
                                  int *nx, int *ny, int *nz);
/* read_variable into a host grid of the variable's type and extents */
ocu_status ocu_nc_reader_read(const ocu_nc_reader *r, const char *name, void *origin, int nc_type, long long xstride,
                              long long ystride, int nx, int ny, int nz, int time_level);

/* ---- persistent refinement ensembles ----------------------------------------------------
 * No reference counterpart as a whole: many Sol_MultigridPressure3DBase::solve calls
 * (sol_mgpressure3d.cpp:332-370: sqrt(sum r^2 / N) of the residual against an absolute
 * tolerance) on right-hand sides of uneven sizes, run as ONE persistent kernel launch (replayed
 * from a CUDA graph).  Each block takes the next member (largest first) from a device counter
 * and runs its whole solve: an FP64 iterative refinement (FP64 residual and pressure) whose
 * corrections are FP32 multigrid solves on the library's red/black split levels (nested
 * iteration + `cycles` V-cycles), until the FP64 residual's L2 norm is at most the member's
 * tolerance or max_outer corrections were applied.  No block waits for another block.
 * Results are checked against FP64 multigrid solutions at the tolerance, not bit for bit. */
typedef struct ocu_pens ocu_pens;
typedef struct ocu_pens_params {
  ocu_bc_set bc;       /* every member's boundary conditions (fixed at creation); faces Neumann,
                          Dirichlet, periodic (even sizes on every level) or none */
  int nu1, nu2;        /* red-black iterations before / after the coarse correction */
  int cycles;          /* V-cycles at level 0 per correction, after the nested iteration
                          (0: the nested iteration alone) */
  int ramp_iters;      /* iterations per level on the way up the nested iteration (0 = nu1+nu2) */
  int max_outer;       /* corrections at most (0 = 10) */
  int threads;         /* threads per block: 256, 512 or 1024 */
  int dense;           /* 1: 1536 threads per SM at up to 42 registers (threads 256 or 512);
                          0: 1024 threads per SM at up to 64 */
  int tail_cells;      /* levels with at most this many cells are solved in shared memory
                          (0 = 512; fixed at creation) */
  double ms;           /* autotuner: measured solve time of the chosen setting */
} ocu_pens_params;
typedef struct ocu_pens_stats {
  int converged;       /* 1 when the last solve reached the member's tolerance */
  int corrections;     /* FP32 correction solves applied */
  int vcycles;         /* level-0 V-cycles run by them */
  double l2;           /* FP64 residual norm sqrt(sum r^2 / N) at the last check */
} ocu_pens_stats;
void ocu_pens_params_default(ocu_pens_params *p);
/* dims: 3 ints per member; h: 3 doubles per member. */
ocu_status ocu_pens_create(int members, const int *dims, const double *h, const ocu_pens_params *params,
                           ocu_pens **out);
void ocu_pens_destroy(ocu_pens *e);
ocu_status ocu_pens_set_stream(ocu_pens *e, ocu_stream s);
/* FP64 views (standard layout, ghost 1) owned by the ensemble; the pressure is the initial guess
 * of the next solve and its result. */
ocu_status ocu_pens_rhs(ocu_pens *e, int member, ocu_grid **out);
ocu_status ocu_pens_pressure(ocu_pens *e, int member, ocu_grid **out);
/* tol: one absolute L2 tolerance per member.  *converged gets the members that reached it;
 * OCU_ERR_NOT_CONVERGED if some did not. */
ocu_status ocu_pens_solve(ocu_pens *e, const double *tol, int *converged);
ocu_status ocu_pens_member_stats(const ocu_pens *e, int member, ocu_pens_stats *stats);
ocu_status ocu_pens_get_params(const ocu_pens *e, ocu_pens_params *p);
ocu_status ocu_pens_set_params(ocu_pens *e, const ocu_pens_params *p);
/* blocks of the persistent launch, threads per block, bytes of the per-block FP32 hierarchies */
ocu_status ocu_pens_launch_shape(const ocu_pens *e, int *blocks, int *threads, long long *scratch_bytes);
/* Times whole solves from a zero guess over thread counts, cycles and smoothing pairs; keeps the
 * fastest that converges every member (ms set); leaves every pressure zeroed. */
ocu_status ocu_pens_autotune(ocu_pens *e, const double *tol);

/* ---- projection (Sol_ProjectDivergence3DDevice<T>, sol_project3d.h:29-129) ------------- */
ocu_status ocu_project_create(ocu_dtype dtype, ocu_project **out);
/* The same with the pressure solver's kind chosen: OCU_MG_F32 / OCU_MG_F64 are
 * Sol_ProjectDivergence3DDevice<float/double> (ocu_project_create); OCU_MG_MIXED_WARMSTART is
 * Sol_ProjectDivergenceMixed3DDeviceD (sol_projectmixed3d.h:28-45, sol_projectmixed3d.cu:24-94:
 * FP64 fields, the reference mixed pressure solver); OCU_MG_MIXED_IR is that class with this
 * library's FP32-in-FP64 refinement solver instead.  The mixed kinds take FP64 grids. */
ocu_status ocu_project_create_with(ocu_mg_kind pressure_kind, ocu_project **out);
/* Field precision and pressure solver chosen separately; besides the combinations above, FP32
 * fields with OCU_MG_MIXED_IR (an FP64 pressure solved by FP32 V-cycles in FP64 refinement,
 * applied to the FP32 velocity in double).  Not a reference class. */
ocu_status ocu_project_create_fields(ocu_dtype fields, ocu_mg_kind pressure_kind, ocu_project **out);
void ocu_project_destroy(ocu_project *p);
ocu_status ocu_project_set_stream(ocu_project *p, ocu_stream s);
/* initialize_storage (sol_project3ddev.cu:100-135): u,v,w borrowed MAC grids of one layout. */
ocu_status ocu_project_initialize_storage(ocu_project *p, int nx, int ny, int nz, double hx,
                                          double hy, double hz, ocu_grid *u, ocu_grid *v,
                                          ocu_grid *w, const ocu_bc_set *bc);
ocu_status ocu_project_solve(ocu_project *p, double tolerance);           /* :58-71 */
ocu_status ocu_project_solve_divergence_only(ocu_project *p);             /* :73-84 */
ocu_grid *ocu_project_divergence(ocu_project *p);
ocu_mg *ocu_project_pressure_solver(ocu_project *p);

/* ---- incompressible Navier-Stokes / Boussinesq (Eqn_IncompressibleNS3D<T>,
 *      ocuequation/eqn_incompressns3d.h:34-248) ------------------------------------------ */
typedef struct ocu_ns_params {
  int nx, ny, nz;
  double hx, hy, hz;
  double max_divergence;
  ocu_bc_set temp_bc;
  ocu_bc_set flow_bc;
  int vertical_direction;        /* ocu_direction */
  double gravity;                /* rounded to T, like the reference's T fields */
  double bouyancy;
  double thermal_diffusion;
  double viscosity;
  int advection_scheme;          /* ocu_interpolation */
  int time_step;                 /* ocu_timestep */
  double cfl_factor;
  int mixed_pressure;            /* not a reference field (0 = the reference's projection): 1 = the
                                    projection's pressure is solved by FP32 V-cycles inside FP64
                                    refinement (FP64 pressure, the fields keep their precision),
                                    which reaches tolerances an FP32 multigrid cannot */
} ocu_ns_params;

/* Eqn_IncompressibleNS3DParams() defaults (eqn_incompressns3d.h:62-73). */
void ocu_ns_params_default(ocu_ns_params *p);
/* Layouts of Eqn_IncompressibleNS3DParams::init_grids (eqn_incompressns3d.h:75-83);
 * which = 'u','v','w','t'. */
ocu_status ocu_ns_init_layout(int nx, int ny, int nz, char which, ocu_layout *out);
ocu_status ocu_ns_create(ocu_dtype dtype, ocu_ns **out);
void ocu_ns_destroy(ocu_ns *ns);
ocu_status ocu_ns_set_stream(ocu_ns *ns, ocu_stream s);
/* set_parameters (eqn_incompressns3d.cu:164-298); init_* are HOST buffers in the
 * init_grids layouts. */
ocu_status ocu_ns_set_parameters(ocu_ns *ns, const ocu_ns_params *params, const void *init_u,
                                 const void *init_v, const void *init_w,
                                 const void *init_temp);
/* get_max_stable_timestep (:301-328); blocks the host for three maxabs reductions. */
ocu_status ocu_ns_get_max_stable_timestep(ocu_ns *ns, double *dt);
/* advance_one_step (:331-399).  The step's work before the projection is replayed as one CUDA
 * graph from the second step of each time-stepping state on (dt is read from device memory, so
 * any dt replays); OCU_B200_NS_GRAPH=0 or OCU_B200_GRAPHS=0 issues it as plain launches.  With
 * the NULL stream the solver works on a private blocking stream (NULL orders against it). */
ocu_status ocu_ns_advance_one_step(ocu_ns *ns, double dt);
ocu_status ocu_ns_advance(ocu_ns *ns, double dt);       /* Equation::advance, equation.cpp:31-56 */
/* get_u/v/w/temperature (:171-174) and the time derivatives 'U','V','W','T', pressure 'p'. */
ocu_grid *ocu_ns_grid(ocu_ns *ns, char which);
int ocu_ns_num_steps(const ocu_ns *ns);

#ifdef __cplusplus
}
#endif

#endif /* OCU_B200_H */
