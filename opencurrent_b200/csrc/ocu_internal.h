// Internal declarations shared by the CUDA translation units of libocu_b200.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>

#include "../../include/ocu_b200.h"

struct ocu_grid {
  ocu_dtype dtype;
  ocu_layout L;
  void *buf;
  bool owned;
};

namespace ocub {

// ---- error reporting (thread-local message behind ocu_last_error) ----------------------
void set_error(const char *fmt, ...);
ocu_status fail(ocu_status st, const char *fmt, ...);
ocu_status check_cuda(cudaError_t e, const char *what);
ocu_status check_launch(const char *what);
void count_launch(int n = 1);
unsigned long long launch_count();
void set_capturing(bool on);
unsigned long long launch_count_captured();
const char *last_error_text();

// ---- programmatic dependent launch ---------------------------------------------------------
// The multigrid, grid and boundary kernels are launched with
// cudaLaunchAttributeProgrammaticStreamSerialization: the next kernel of a stream may be
// scheduled while its predecessor is still running.  Every kernel launched this way starts with
// pdl_entry(): griddepcontrol.wait returns once the predecessor grid has completed and its
// memory operations are visible, so nothing is read or written before that; the
// launch_dependents that follows lets the successor's blocks be scheduled early.  A kernel
// launched without the attribute passes the wait at once.  OCU_B200_PDL=0 turns the attribute off.
bool pdl_enabled();
// Launches on several concurrent streams (ensemble classes) go without the attribute: a
// successor's early-scheduled blocks would hold SM slots the other streams' kernels could use.
bool pdl_suppressed();
void set_pdl_suppressed(bool on);
struct PdlSuppress {
  bool prev;
  PdlSuppress() : prev(pdl_suppressed()) { set_pdl_suppressed(true); }
  ~PdlSuppress() { set_pdl_suppressed(prev); }
};

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args &&...args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = (pdl_enabled() && !pdl_suppressed()) ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

#ifdef __CUDACC__
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#endif

inline size_t dtype_size(ocu_dtype d) { return d == OCU_F64 ? 8 : 4; }

template <typename T> inline T *origin(ocu_grid *g) { return static_cast<T *>(g->buf) + g->L.shift; }
template <typename T> inline const T *origin(const ocu_grid *g) { return static_cast<const T *>(g->buf) + g->L.shift; }

inline bool layout_match(const ocu_layout &a, const ocu_layout &b) {
  return a.pnx == b.pnx && a.pny == b.pny && a.pnz == b.pnz;
}

void layout_compute(int nx, int ny, int nz, int gx, int gy, int gz, int padx, int pady, int padz,
                    ocu_layout *L);

// Face-by-face view of a BoundaryConditionSet for kernels (passed by value).
struct BCDev {
  int type[6];     // xpos, xneg, ypos, yneg, zpos, zneg
  float value[6];
  float aux[6];
  // Per-face reads by a run-time face index, as select chains: indexing the arrays directly
  // with a non-constant index makes every thread copy the struct to local memory.
  __host__ __device__ __forceinline__ int ty(int f) const {
    return f == 0 ? type[0] : f == 1 ? type[1] : f == 2 ? type[2] : f == 3 ? type[3] : f == 4 ? type[4] : type[5];
  }
  __host__ __device__ __forceinline__ float val(int f) const {
    return f == 0 ? value[0] : f == 1 ? value[1] : f == 2 ? value[2] : f == 3 ? value[3] : f == 4 ? value[4] : value[5];
  }
  __host__ __device__ __forceinline__ float auxv(int f) const {
    return f == 0 ? aux[0] : f == 1 ? aux[1] : f == 2 ? aux[2] : f == 3 ? aux[3] : f == 4 ? aux[4] : aux[5];
  }
};
BCDev to_dev(const ocu_bc_set &bc);
bool bc_check_scalar(const ocu_bc_set &bc);
bool bc_check_mac(const ocu_bc_set &bc);
bool bc_any_periodic(const ocu_bc_set &bc);
void bc_make_homogeneous(ocu_bc_set *bc);
double bc_diag_mod(const ocu_bc &b, double factor);
bool check_float(float f);

// ---- launchers (kernels_*.cu) -----------------------------------------------------------
// Every launcher enqueues on stream s and returns OCU_OK or an error from the launch.
template <typename T>
ocu_status launch_bc_level1(T *origin, const ocu_layout &L, const ocu_bc_set &bc, double hx,
                            double hy, double hz, cudaStream_t s);
template <typename T>
ocu_status launch_bc_nocorners_dev(T *origin, const ocu_layout &L, const ocu_bc_set &bc,
                                   double hx, double hy, double hz, cudaStream_t s);
template <typename T>
ocu_status launch_mac_bc_level1(T *u, T *v, T *w, const ocu_layout &L, int nx, int ny, int nz,
                                const ocu_bc_set &bc, cudaStream_t s);

template <typename T>
ocu_status launch_clear(T *buf, long long n, T value, cudaStream_t s);
template <typename T, typename S>
ocu_status launch_convert(T *dst, const S *src, long long n, cudaStream_t s);
template <typename T>
ocu_status launch_lincomb1(T *res, T a1, const T *g1, long long n, cudaStream_t s);
// A coefficient of a linear-combination kernel: the value itself, or (p set) the value the
// kernel reads from device memory after its programmatic-dependency wait -- so a launch captured
// once in a CUDA graph takes a new time step at every replay.
template <typename T>
struct Coef {
  T v;
  const T *p;
  __host__ __device__ Coef(T value) : v(value), p(nullptr) {}
  __host__ __device__ Coef(T value, const T *ptr) : v(value), p(ptr) {}
#ifdef __CUDACC__
  __device__ __forceinline__ T get() const { return p ? *p : v; }
#endif
};
template <typename T>
ocu_status launch_lincomb2(T *res, const ocu_layout &L, T a1, const T *g1, Coef<T> a2, const T *g2,
                           cudaStream_t s);

// Reduction in the reference fold order over the interior of a grid; the T result is stored
// as double at *d_result (device pointer).  d_scratch: >= reduce_scratch_elems(L) elements of
// T plus one unsigned counter (see kernels_grid.cu).
size_t reduce_scratch_bytes(const ocu_layout &L, size_t elem);
// n <= 32 doubles from device memory into pinned (cudaMallocHost) host memory by a kernel's
// stores instead of a copy-engine transfer (see kernels_grid.cu)
ocu_status launch_readback(const double *src, double *host_pinned, int n, cudaStream_t s);
// min, max or max-abs (op) of n <= 3 grids sharing strides, one launch, into results[0..n)
template <typename T>
ocu_status launch_minmax(const T *const *origins, const ocu_layout *const *lays, int n, int op, void *d_scratch,
                         double *d_results, cudaStream_t s);
template <typename T>
ocu_status launch_dot(const T *a, const T *b, const ocu_layout &L, void *d_scratch, double *d_result, cudaStream_t s);
template <typename T>
ocu_status launch_reduce(const T *origin, const ocu_layout &L, int op, void *d_scratch,
                         double *d_result, cudaStream_t s);

// ---- multigrid level operations (kernels_mg.cu) ------------------------------------------
struct RelaxParams {
  double omega, h, fx, fy, fz;
  ocu_bc_set bc;   // bc at this level
};
template <typename T>
ocu_status launch_relax_color(T *u, const T *b, const ocu_layout &L, const T *diag, int color,
                              const RelaxParams &p, cudaStream_t s);
template <typename T>
ocu_status launch_init_diag(T *diag, int nx, int ny, const RelaxParams &p, cudaStream_t s);
// Coarsest-level relaxation with the host routine's arithmetic and ghost handling
// (sol_mgpressure3ddev.cu:82-188), as one single-CTA kernel.
template <typename T>
ocu_status launch_coarse_relax(T *u, const T *b, const ocu_layout &L, int iterations, int order,
                               const RelaxParams &p, double hx, double hy, double hz,
                               cudaStream_t s);
template <typename T>
ocu_status launch_residual(const T *u, const T *b, T *r, const ocu_layout &L, double h,
                           double fx, double fy, double fz, cudaStream_t s);
template <typename T>
ocu_status launch_restrict(const T *r, const ocu_layout &Lf, T *bc_, const ocu_layout &Lc,
                           cudaStream_t s);
template <typename T>
ocu_status launch_prolong(const T *uc, const ocu_layout &Lc, T *uf, const ocu_layout &Lf,
                          cudaStream_t s);
// IR helpers: r32 = (float) r64 on the interior; x64 += (double) e32 on the interior.
ocu_status launch_downcast_interior(const double *r, float *b32, const ocu_layout &L,
                                    cudaStream_t s);
ocu_status launch_add_correction(double *x, const float *e, const ocu_layout &L,
                                 cudaStream_t s);

// ---- flow stencils (kernels_flow.cu) ---------------------------------------------------------
template <typename T>
ocu_status launch_divergence(const T *u, const T *v, const T *w, T *div, const ocu_layout &L,
                             int nx, int ny, int nz, double hx, double hy, double hz,
                             cudaStream_t s);
template <typename T>
ocu_status launch_gradient(T *u, T *v, T *w, const T *phi, const ocu_layout &L, int nx, int ny,
                           int nz, double hx, double hy, double hz, T coefficient,
                           cudaStream_t s);
// u, v, w (float) -= c grad(phi) with phi in double
ocu_status launch_gradient_p64(float *u, float *v, float *w, const double *phi, const ocu_layout &L, int nx, int ny,
                              int nz, double hx, double hy, double hz, double coefficient, cudaStream_t s);
// u, v, w (one layout) += a2 d [then += a3 l]: one launch, or OCU_ERR_UNSUPPORTED
template <typename T>
ocu_status launch_update3(T *const *x, const T *const *d, const T *const *l, const ocu_layout &L, Coef<T> a2,
                          Coef<T> a3, cudaStream_t s);
// diffusion + buoyancy of the vertical velocity in one pass (FP32), or OCU_ERR_UNSUPPORTED
ocu_status launch_laplacian_thermal(const float *phi, float *dphidt, const ocu_layout &L, int nx, int ny, int nz,
                                    double hx, double hy, double hz, float coefficient, const float *temp, float ct,
                                    long long nbr, int tnx, int tny, int tnz, cudaStream_t s);
template <typename T>
ocu_status launch_laplacian(const T *phi, T *dphidt, const ocu_layout &L, int nx, int ny,
                            int nz, double hx, double hy, double hz, T coefficient,
                            cudaStream_t s);
template <typename T>
ocu_status launch_advect_self(const T *u, const T *v, const T *w, T *du, T *dv, T *dw,
                              const ocu_layout &L, int nx, int ny, int nz, double hx, double hy,
                              double hz, int interp, cudaStream_t s);
template <typename T>
ocu_status launch_advect_passive(const T *u, const T *v, const T *w, const T *phi, T *dphi,
                                 const ocu_layout &L, int nx, int ny, int nz, double hx,
                                 double hy, double hz, int interp, cudaStream_t s);
// FP32 self-advection fed by TMA (kernels_flow.cu), bit-identical to launch_advect_self;
// OCU_ERR_UNSUPPORTED where it does not apply (the caller then uses launch_advect_self).  err:
// device word set when a load wait gives up (nullptr: never taken); wait_limit: polls per wait
// (0: the default; negative: the timeout test, a first wait that nothing completes).
ocu_status launch_advect_self_tma(const float *u, const float *v, const float *w, float *du, float *dv,
                                  float *dw, const ocu_layout &L, int nx, int ny, int nz, double hx,
                                  double hy, double hz, int interp, int *err, int wait_limit,
                                  cudaStream_t s);
template <typename T>
ocu_status launch_thermal_force(T *dvdt, T coefficient, const T *temp, const ocu_layout &L,
                                int nbr_stride, int nx, int ny, int nz, cudaStream_t s);

}  // namespace ocub

#define OCU_TRY(...)                         \
  do {                                       \
    ocu_status _st = (__VA_ARGS__);          \
    if (_st != OCU_OK) return _st;           \
  } while (0)
