// Flow stencils on the MAC grid: divergence, gradient update, centred Laplacian, upwind /
// centred self-advection and passive-scalar advection, Boussinesq buoyancy.
//
// All grids handed to one kernel share a padded layout (the reference requires it,
// sol_selfadvection3ddev.cu:616-620), so one index serves every array.  Expression order is
// the reference's; built with --fmad=false.
#include "ocu_internal.h"

namespace ocub {

// A thread visits CI cells along i (the same k, j): their loads are independent, so they are in
// flight together, and a plane's values serve the neighbouring cells as well.  The light
// stencils take kCellsI; self-advection, which is bound by instruction issue, takes one.
constexpr int kCellsI = 4;

static inline void shape(int nx, int ny, int nz, dim3 *grid, dim3 *block, int ci = kCellsI) {
  *block = nz >= 64 ? dim3(64, 4) : dim3(32, 8);
  *grid = dim3((nz + block->x - 1) / block->x, (ny + block->y - 1) / block->y, (nx + ci - 1) / ci);
}

#define CELL_LOOP_BEGIN_CI(CI)                                    \
  const int k = blockIdx.x * blockDim.x + threadIdx.x;            \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;            \
  if (k >= nz || j >= ny) return;                                 \
  _Pragma("unroll") for (int ci = 0; ci < (CI); ci++) {           \
    const int i = blockIdx.z * (CI) + ci;                         \
    if (i >= nx) break;                                           \
    const long long id = (long long)i * xs + (long long)j * ys + k;
#define CELL_LOOP_BEGIN CELL_LOOP_BEGIN_CI(kCellsI)
#define CELL_LOOP_END }

// Sol_Divergence3DDevice_calculate_divergence (sol_divergence3ddev.cu:23-45)
template <typename T>
__global__ void k_divergence(const T *__restrict__ u, const T *__restrict__ v, const T *__restrict__ w,
                             T *__restrict__ div, T ihx, T ihy, T ihz, long long xs, long long ys, int nx, int ny,
                             int nz) {
  CELL_LOOP_BEGIN
  div[id] = ihx * (u[id + xs] - u[id]) + ihy * (v[id + ys] - v[id]) + ihz * (w[id + 1] - w[id]);
  CELL_LOOP_END
}

// Sol_Gradient3DDevice_subtract_grad (sol_gradient3ddev.cu:24-47)
template <typename T>
__global__ void k_gradient(T *__restrict__ u, T *__restrict__ v, T *__restrict__ w, const T *__restrict__ phi,
                           T c, T ihx, T ihy, T ihz, long long xs, long long ys, int nx, int ny, int nz) {
  CELL_LOOP_BEGIN
  const T p = phi[id];
  u[id] += c * ihx * (p - phi[id - xs]);
  v[id] += c * ihy * (p - phi[id - ys]);
  w[id] += c * ihz * (p - phi[id - 1]);
  CELL_LOOP_END
}

// The same update with the pressure in double and the velocity in T: the difference and the
// update in double, rounded to T once (the projection with a refinement-solved FP64 pressure).
template <typename T>
__global__ void k_gradient_p64(T *__restrict__ u, T *__restrict__ v, T *__restrict__ w, const double *__restrict__ phi,
                               double c, double ihx, double ihy, double ihz, long long xs, long long ys, int nx, int ny,
                               int nz) {
  CELL_LOOP_BEGIN
  const double p = phi[id];
  u[id] = (T)((double)u[id] + c * ihx * (p - phi[id - xs]));
  v[id] = (T)((double)v[id] + c * ihy * (p - phi[id - ys]));
  w[id] = (T)((double)w[id] + c * ihz * (p - phi[id - 1]));
  CELL_LOOP_END
}

// Sol_LaplacianCentered3DDevice_stencil (sol_laplaciancent3ddev.cu:28-60)
template <typename T>
__global__ void k_laplacian(const T *__restrict__ phi, T *__restrict__ dphidt, T ihx2, T ihy2, T ihz2, T c,
                            long long xs, long long ys, int nx, int ny, int nz) {
  CELL_LOOP_BEGIN
  const T p = phi[id];
  const T d = dphidt[id];
  const T lap = ihz2 * (phi[id + 1] + phi[id - 1] - ((T)2) * p) + ihy2 * (phi[id + ys] + phi[id - ys] - ((T)2) * p) +
                ihx2 * (phi[id + xs] + phi[id - xs] - ((T)2) * p);
  dphidt[id] = d + c * lap;
  CELL_LOOP_END
}

// InterpolatorFirstOrderUpwind / InterpolatorSecondOrderCentered (interpolation.h:35-48)
template <typename T, int IT>
__device__ __forceinline__ T interp(T u, T x0, T x1) {
  if (IT == OCU_IT_FIRST_ORDER_UPWIND) return u < 0 ? x1 : x0;
  return ((T)0.5) * (x1 + x0);
}

// Advection3DF/D_apply_upwind_TEX (sol_selfadvection3ddev.cu:135-337)
template <typename T, int IT>
__global__ void __launch_bounds__(256) k_advect_self(const T *__restrict__ u, const T *__restrict__ v,
                                                     const T *__restrict__ w, T *__restrict__ dudt,
                                                     T *__restrict__ dvdt, T *__restrict__ dwdt, T ihx, T ihy,
                                                     T ihz, long long xs, long long ys, int nx, int ny, int nz) {
  CELL_LOOP_BEGIN_CI(1)
  const T half = (T)0.5;
  const long long pi = id + xs, pj = id + ys, pk = id + 1, mi = id - xs, mj = id - ys, mk = id - 1;
  const T ui = u[id], vi = v[id], wi = w[id];
  T a, b, d1, d2, d3;
  a = half * (ui + u[pi]);
  b = half * (ui + u[mi]);
  d1 = (a * interp<T, IT>(a, ui, u[pi])) - (b * interp<T, IT>(b, u[mi], ui));
  a = half * (v[pj] + v[pj - xs]);
  b = half * (vi + v[mi]);
  d2 = (a * interp<T, IT>(a, ui, u[pj])) - (b * interp<T, IT>(b, u[mj], ui));
  a = half * (w[pk] + w[pk - xs]);
  b = half * (wi + w[mi]);
  d3 = (a * interp<T, IT>(a, ui, u[pk])) - (b * interp<T, IT>(b, u[mk], ui));
  dudt[id] = -d1 * ihx - d2 * ihy - d3 * ihz;

  a = half * (u[pi] + u[pi - ys]);
  b = half * (ui + u[mj]);
  d1 = (a * interp<T, IT>(a, vi, v[pi])) - (b * interp<T, IT>(b, v[mi], vi));
  a = half * (vi + v[pj]);
  b = half * (vi + v[mj]);
  d2 = (a * interp<T, IT>(a, vi, v[pj])) - (b * interp<T, IT>(b, v[mj], vi));
  a = half * (w[pk] + w[pk - ys]);
  b = half * (wi + w[mj]);
  d3 = (a * interp<T, IT>(a, vi, v[pk])) - (b * interp<T, IT>(b, v[mk], vi));
  dvdt[id] = -d1 * ihx - d2 * ihy - d3 * ihz;

  a = half * (u[pi] + u[pi - 1]);
  b = half * (ui + u[mk]);
  d1 = (a * interp<T, IT>(a, wi, w[pi])) - (b * interp<T, IT>(b, w[mi], wi));
  a = half * (v[pj] + v[pj - 1]);
  b = half * (vi + v[mk]);
  d2 = (a * interp<T, IT>(a, wi, w[pj])) - (b * interp<T, IT>(b, w[mj], wi));
  a = half * (wi + w[pk]);
  b = half * (wi + w[mk]);
  d3 = (a * interp<T, IT>(a, wi, w[pk])) - (b * interp<T, IT>(b, w[mk], wi));
  dwdt[id] = -d1 * ihx - d2 * ihy - d3 * ihz;
  CELL_LOOP_END
}

// Sol_PassiveAdvection3D_apply_interp (sol_passiveadvection3ddev.cu:31-78)
template <typename T, int IT>
__global__ void __launch_bounds__(256) k_advect_passive(const T *__restrict__ u, const T *__restrict__ v,
                                                        const T *__restrict__ w, const T *__restrict__ phi,
                                                        T *__restrict__ dphidt, T ihx, T ihy, T ihz, long long xs,
                                                        long long ys, int nx, int ny, int nz) {
  CELL_LOOP_BEGIN
  const T p = phi[id];
  const T upi = u[id + xs], uij = u[id];
  const T du = upi * interp<T, IT>(upi, p, phi[id + xs]) - uij * interp<T, IT>(uij, phi[id - xs], p);
  const T vpj = v[id + ys], vij = v[id];
  const T dv = vpj * interp<T, IT>(vpj, p, phi[id + ys]) - vij * interp<T, IT>(vij, phi[id - ys], p);
  const T wpk = w[id + 1], wij = w[id];
  const T dw = wpk * interp<T, IT>(wpk, p, phi[id + 1]) - wij * interp<T, IT>(wij, phi[id - 1], p);
  dphidt[id] = (-du * ihx) - (dv * ihy) - (dw * ihz);
  CELL_LOOP_END
}

// Eqn_IncompressibleNS3D_add_thermal_force (eqn_incompressns3d.cu:25-44)
template <typename T>
__global__ void k_thermal_force(T *__restrict__ dvdt, T c, const T *__restrict__ temp, long long nbr, long long xs,
                                long long ys, int nx, int ny, int nz) {
  CELL_LOOP_BEGIN
  dvdt[id] += ((T)0.5) * c * (temp[id] + temp[id - nbr]);
  CELL_LOOP_END
}

template <typename T>
ocu_status launch_divergence(const T *u, const T *v, const T *w, T *div, const ocu_layout &L,
                             int nx, int ny, int nz, double hx, double hy, double hz,
                             cudaStream_t s) {
  dim3 g, b;
  shape(nx, ny, nz, &g, &b);
  k_divergence<T><<<g, b, 0, s>>>(u, v, w, div, (T)(1 / hx), (T)(1 / hy), (T)(1 / hz), L.xstride, L.ystride, nx,
                                  ny, nz);
  return check_launch("k_divergence");
}

template <typename T>
ocu_status launch_gradient(T *u, T *v, T *w, const T *phi, const ocu_layout &L, int nx, int ny,
                           int nz, double hx, double hy, double hz, T coefficient,
                           cudaStream_t s) {
  dim3 g, b;
  shape(nx, ny, nz, &g, &b);
  k_gradient<T><<<g, b, 0, s>>>(u, v, w, phi, coefficient, (T)(1 / hx), (T)(1 / hy), (T)(1 / hz), L.xstride,
                                L.ystride, nx, ny, nz);
  return check_launch("k_gradient");
}

ocu_status launch_gradient_p64(float *u, float *v, float *w, const double *phi, const ocu_layout &L, int nx, int ny,
                              int nz, double hx, double hy, double hz, double coefficient, cudaStream_t s) {
  dim3 g, b;
  shape(nx, ny, nz, &g, &b);
  k_gradient_p64<float><<<g, b, 0, s>>>(u, v, w, phi, coefficient, 1 / hx, 1 / hy, 1 / hz, L.xstride, L.ystride, nx,
                                        ny, nz);
  return check_launch("k_gradient_p64");
}

template <typename T>
ocu_status launch_laplacian(const T *phi, T *dphidt, const ocu_layout &L, int nx, int ny,
                            int nz, double hx, double hy, double hz, T coefficient,
                            cudaStream_t s) {
  dim3 g, b;
  shape(nx, ny, nz, &g, &b);
  k_laplacian<T><<<g, b, 0, s>>>(phi, dphidt, (T)(1 / (hx * hx)), (T)(1 / (hy * hy)), (T)(1 / (hz * hz)),
                                 coefficient, L.xstride, L.ystride, nx, ny, nz);
  return check_launch("k_laplacian");
}

template <typename T>
ocu_status launch_advect_self(const T *u, const T *v, const T *w, T *du, T *dv, T *dw,
                              const ocu_layout &L, int nx, int ny, int nz, double hx, double hy,
                              double hz, int it, cudaStream_t s) {
  dim3 g, b;
  shape(nx, ny, nz, &g, &b, 1);
  const T ihx = (T)(1 / hx), ihy = (T)(1 / hy), ihz = (T)(1 / hz);
  if (it == OCU_IT_FIRST_ORDER_UPWIND)
    k_advect_self<T, OCU_IT_FIRST_ORDER_UPWIND><<<g, b, 0, s>>>(u, v, w, du, dv, dw, ihx, ihy, ihz, L.xstride,
                                                               L.ystride, nx, ny, nz);
  else if (it == OCU_IT_SECOND_ORDER_CENTERED)
    k_advect_self<T, OCU_IT_SECOND_ORDER_CENTERED><<<g, b, 0, s>>>(u, v, w, du, dv, dw, ihx, ihy, ihz, L.xstride,
                                                                  L.ystride, nx, ny, nz);
  else
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_SelfAdvection3DDevice::solve_tex - invalid interpolation type %d", it);
  return check_launch("k_advect_self");
}

template <typename T>
ocu_status launch_advect_passive(const T *u, const T *v, const T *w, const T *phi, T *dphi,
                                 const ocu_layout &L, int nx, int ny, int nz, double hx,
                                 double hy, double hz, int it, cudaStream_t s) {
  dim3 g, b;
  shape(nx, ny, nz, &g, &b);
  const T ihx = (T)(1 / hx), ihy = (T)(1 / hy), ihz = (T)(1 / hz);
  if (it == OCU_IT_FIRST_ORDER_UPWIND)
    k_advect_passive<T, OCU_IT_FIRST_ORDER_UPWIND><<<g, b, 0, s>>>(u, v, w, phi, dphi, ihx, ihy, ihz, L.xstride,
                                                                  L.ystride, nx, ny, nz);
  else if (it == OCU_IT_SECOND_ORDER_CENTERED)
    k_advect_passive<T, OCU_IT_SECOND_ORDER_CENTERED><<<g, b, 0, s>>>(u, v, w, phi, dphi, ihx, ihy, ihz,
                                                                     L.xstride, L.ystride, nx, ny, nz);
  else
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_PassiveAdvection3DDevice::solve() - invalid interpolation type %d", it);
  return check_launch("k_advect_passive");
}

template <typename T>
ocu_status launch_thermal_force(T *dvdt, T coefficient, const T *temp, const ocu_layout &L,
                                int nbr_stride, int nx, int ny, int nz, cudaStream_t s) {
  dim3 g, b;
  shape(nx, ny, nz, &g, &b);
  k_thermal_force<T><<<g, b, 0, s>>>(dvdt, coefficient, temp, nbr_stride, L.xstride, L.ystride, nx, ny, nz);
  return check_launch("k_thermal_force");
}

#define INST(T)                                                                                          \
  template ocu_status launch_divergence<T>(const T *, const T *, const T *, T *, const ocu_layout &, int, \
                                           int, int, double, double, double, cudaStream_t);             \
  template ocu_status launch_gradient<T>(T *, T *, T *, const T *, const ocu_layout &, int, int, int,     \
                                         double, double, double, T, cudaStream_t);                      \
  template ocu_status launch_laplacian<T>(const T *, T *, const ocu_layout &, int, int, int, double,      \
                                          double, double, T, cudaStream_t);                             \
  template ocu_status launch_advect_self<T>(const T *, const T *, const T *, T *, T *, T *,               \
                                            const ocu_layout &, int, int, int, double, double, double,  \
                                            int, cudaStream_t);                                         \
  template ocu_status launch_advect_passive<T>(const T *, const T *, const T *, const T *, T *,           \
                                               const ocu_layout &, int, int, int, double, double,       \
                                               double, int, cudaStream_t);                              \
  template ocu_status launch_thermal_force<T>(T *, T, const T *, const ocu_layout &, int, int, int, int,  \
                                              cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace ocub
