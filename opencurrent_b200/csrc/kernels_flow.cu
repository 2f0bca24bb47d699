// Flow stencils on the MAC grid: divergence, gradient update, centred Laplacian, upwind /
// centred self-advection and passive-scalar advection, Boussinesq buoyancy.
//
// All grids handed to one kernel share a padded layout (the reference requires it,
// sol_selfadvection3ddev.cu:616-620), so one index serves every array.  Expression order is
// the reference's; built with --fmad=false.
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <initializer_list>

#include "ocu_internal.h"
#include "tma_ptx.cuh"

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

// ---- FP32 forms on 16-byte groups along k ---------------------------------------------------
// A thread owns four consecutive cells of a row (one float4) at CI consecutive i; its z
// neighbours k - 1 and k + 4 come from the adjacent lanes (warp shuffles), the first / last
// group of a block row loads them itself.  Each cell's expression is the scalar kernel's, in its
// order, so results are bit-identical; only the loads are wider (a quarter of the load
// instructions, 16-byte transactions).  Used when nz, both strides and the interior origin are
// multiples of four floats.
#ifndef OCU_FLOW_CELLS_I
#define OCU_FLOW_CELLS_I 4
#endif
constexpr int kCellsIV = OCU_FLOW_CELLS_I;

struct Row4 {
  float v[6];  // cells k - 1 .. k + 4
};

__device__ __forceinline__ float4 ld4g(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4g(float *p, float a, float b, float c, float d) {
  *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, d);
}

// the group at id with its k - 1 and k + 4 neighbours; every lane of the warp calls it
__device__ __forceinline__ Row4 row4(const float *__restrict__ p, long long id, bool ok, bool first, bool last) {
  const float4 c = ok ? ld4g(p + id) : make_float4(0.f, 0.f, 0.f, 0.f);
  Row4 r;
  r.v[1] = c.x; r.v[2] = c.y; r.v[3] = c.z; r.v[4] = c.w;
  r.v[0] = __shfl_up_sync(0xffffffffu, c.w, 1);
  r.v[5] = __shfl_down_sync(0xffffffffu, c.x, 1);
  if (ok && first) r.v[0] = p[id - 1];
  if (ok && last) r.v[5] = p[id + 4];
  return r;
}

#define V4_BEGIN_CI(CI)                                                                          \
  const int k4 = blockIdx.x * blockDim.x + threadIdx.x;                                          \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;                                           \
  const bool ok = k4 < nz4 && j < ny;                                                            \
  const bool first = threadIdx.x == 0, last = threadIdx.x == blockDim.x - 1 || k4 == nz4 - 1;    \
  _Pragma("unroll") for (int ci = 0; ci < (CI); ci++) {                                           \
    const int i = blockIdx.z * (CI) + ci;                                                        \
    if (i >= nx) break;                                                                          \
    const long long id = (long long)i * xs + (long long)j * ys + 4 * k4;
#define V4_BEGIN V4_BEGIN_CI(kCellsIV)
#define V4_END }
// Cells per thread along i of the passive advection's group form: one (measured at
// 256x256x128: 35.8 us against 39.8 with four; the other group kernels measured best at four).
constexpr int kCellsIPassive = 1;

// nr (0..3): cells past the last group of a row (rows of nz = 4 nz4 + nr cells); the lane of the
// last group computes them with the scalar expression.
// nr (0..3): cells past the last group of a row (rows of nz = 4 nz4 + nr cells); the blocks
// holding the rows' last groups compute them afterwards, one cell per thread, with the scalar
// expression (handled by the last lane of each row they measured slower: its warp waited).
// TH: the buoyancy term of the same component added after the diffusion term, in the order of
// the reference's two kernels (d + c lap, then + 0.5 ct (T + T_nbr)), on the cells i < tnx,
// j < tny, k < tnz (the temperature's extent; the velocity component has one face layer more).
struct ThermalArgs {
  const float *temp;
  float ct;
  long long nbr;
  int tnx, tny, tnz;
};

template <bool TH>
__global__ void __launch_bounds__(256) k_laplacian_v4(const float *__restrict__ phi, float *__restrict__ dphidt,
                                                      float ihx2, float ihy2, float ihz2, float c, long long xs,
                                                      long long ys, int nx, int ny, int nz4, int nr, ThermalArgs th) {
  if (nr > 0 && blockIdx.x == gridDim.x - 1) {
    const int nt = blockDim.x * blockDim.y, cnt = nr * blockDim.y * kCellsIV;
    for (int t = threadIdx.y * blockDim.x + threadIdx.x; t < cnt; t += nt) {
      const int e = t % nr, ry = (t / nr) % blockDim.y, cr = t / (nr * blockDim.y);
      const int jr = blockIdx.y * blockDim.y + ry, ir = blockIdx.z * kCellsIV + cr;
      if (jr >= ny || ir >= nx) continue;
      const long long q = (long long)ir * xs + (long long)jr * ys + 4 * nz4 + e;
      const float p = phi[q];
      const float lap = ihz2 * (phi[q + 1] + phi[q - 1] - 2.f * p) + ihy2 * (phi[q + ys] + phi[q - ys] - 2.f * p) +
                        ihx2 * (phi[q + xs] + phi[q - xs] - 2.f * p);
      float o = dphidt[q] + c * lap;
      if (TH && ir < th.tnx && jr < th.tny && 4 * nz4 + e < th.tnz)
        o += 0.5f * th.ct * (th.temp[q] + th.temp[q - th.nbr]);
      dphidt[q] = o;
    }
  }
  V4_BEGIN
  const Row4 P = row4(phi, id, ok, first, last);
  // the temperature group (its k - 1 neighbour from the lanes when the vertical is z)
  Row4 TT;
  if (TH) TT = row4(th.temp, id, ok && i < th.tnx && j < th.tny, first, last);
  if (!ok) continue;
  const float4 D = ld4g(dphidt + id), YP = ld4g(phi + id + ys), YM = ld4g(phi + id - ys);
  const float4 XP = ld4g(phi + id + xs), XM = ld4g(phi + id - xs);
  const float yp[4] = {YP.x, YP.y, YP.z, YP.w}, ym[4] = {YM.x, YM.y, YM.z, YM.w};
  const float xp[4] = {XP.x, XP.y, XP.z, XP.w}, xm[4] = {XM.x, XM.y, XM.z, XM.w};
  const float d[4] = {D.x, D.y, D.z, D.w};
  float o[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const float p = P.v[e + 1];
    const float lap = ihz2 * (P.v[e + 2] + P.v[e] - 2.f * p) + ihy2 * (yp[e] + ym[e] - 2.f * p) +
                      ihx2 * (xp[e] + xm[e] - 2.f * p);
    o[e] = d[e] + c * lap;
  }
  if (TH && i < th.tnx && j < th.tny) {
    float t1[4];
    if (th.nbr == 1) {
#pragma unroll
      for (int e = 0; e < 4; e++) t1[e] = TT.v[e];
    } else {  // a multiple of 4: a whole group
      const float4 T1 = ld4g(th.temp + id - th.nbr);
      t1[0] = T1.x; t1[1] = T1.y; t1[2] = T1.z; t1[3] = T1.w;
    }
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (4 * k4 + e < th.tnz) o[e] += 0.5f * th.ct * (TT.v[e + 1] + t1[e]);
  }
  st4g(dphidt + id, o[0], o[1], o[2], o[3]);
  V4_END
}

__global__ void __launch_bounds__(256) k_divergence_v4(const float *__restrict__ u, const float *__restrict__ v,
                                                       const float *__restrict__ w, float *__restrict__ div,
                                                       float ihx, float ihy, float ihz, long long xs, long long ys,
                                                       int nx, int ny, int nz4) {
  V4_BEGIN
  const Row4 W = row4(w, id, ok, first, last);
  if (!ok) continue;
  const float4 U = ld4g(u + id), UP = ld4g(u + id + xs), V = ld4g(v + id), VP = ld4g(v + id + ys);
  const float uu[4] = {U.x, U.y, U.z, U.w}, up[4] = {UP.x, UP.y, UP.z, UP.w};
  const float vv[4] = {V.x, V.y, V.z, V.w}, vp[4] = {VP.x, VP.y, VP.z, VP.w};
  float o[4];
#pragma unroll
  for (int e = 0; e < 4; e++) o[e] = ihx * (up[e] - uu[e]) + ihy * (vp[e] - vv[e]) + ihz * (W.v[e + 2] - W.v[e + 1]);
  st4g(div + id, o[0], o[1], o[2], o[3]);
  V4_END
}

__global__ void __launch_bounds__(256) k_gradient_v4(float *__restrict__ u, float *__restrict__ v,
                                                     float *__restrict__ w, const float *__restrict__ phi, float c,
                                                     float ihx, float ihy, float ihz, long long xs, long long ys,
                                                     int nx, int ny, int nz4) {
  V4_BEGIN
  const Row4 P = row4(phi, id, ok, first, last);
  if (!ok) continue;
  const float4 XM = ld4g(phi + id - xs), YM = ld4g(phi + id - ys);
  const float4 U = ld4g(u + id), V = ld4g(v + id), W = ld4g(w + id);
  const float xm[4] = {XM.x, XM.y, XM.z, XM.w}, ym[4] = {YM.x, YM.y, YM.z, YM.w};
  float uu[4] = {U.x, U.y, U.z, U.w}, vv[4] = {V.x, V.y, V.z, V.w}, ww[4] = {W.x, W.y, W.z, W.w};
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const float p = P.v[e + 1];
    uu[e] += c * ihx * (p - xm[e]);
    vv[e] += c * ihy * (p - ym[e]);
    ww[e] += c * ihz * (p - P.v[e]);
  }
  st4g(u + id, uu[0], uu[1], uu[2], uu[3]);
  st4g(v + id, vv[0], vv[1], vv[2], vv[3]);
  st4g(w + id, ww[0], ww[1], ww[2], ww[3]);
  V4_END
}

// the vertical neighbour along k (nbr = 1) from the lanes, or a whole group (nbr a multiple of 4)
__global__ void __launch_bounds__(256) k_thermal_force_v4(float *__restrict__ dvdt, float c,
                                                          const float *__restrict__ temp, long long nbr,
                                                          long long xs, long long ys, int nx, int ny, int nz4) {
  V4_BEGIN
  const Row4 Tc = row4(temp, id, ok, first, last);
  if (!ok) continue;
  float tn[4];
  if (nbr == 1) {
#pragma unroll
    for (int e = 0; e < 4; e++) tn[e] = Tc.v[e];
  } else {
    const float4 N = ld4g(temp + id - nbr);
    tn[0] = N.x; tn[1] = N.y; tn[2] = N.z; tn[3] = N.w;
  }
  const float4 D = ld4g(dvdt + id);
  float d[4] = {D.x, D.y, D.z, D.w};
#pragma unroll
  for (int e = 0; e < 4; e++) d[e] += 0.5f * c * (Tc.v[e + 1] + tn[e]);
  st4g(dvdt + id, d[0], d[1], d[2], d[3]);
  V4_END
}

template <int IT>
__global__ void __launch_bounds__(256) k_advect_passive_v4(const float *__restrict__ u, const float *__restrict__ v,
                                                           const float *__restrict__ w, const float *__restrict__ phi,
                                                           float *__restrict__ dphidt, float ihx, float ihy, float ihz,
                                                           long long xs, long long ys, int nx, int ny, int nz4) {
  V4_BEGIN_CI(kCellsIPassive)
  const Row4 P = row4(phi, id, ok, first, last);
  const Row4 W = row4(w, id, ok, first, last);
  if (!ok) continue;
  const float4 UP = ld4g(u + id + xs), U = ld4g(u + id), PXP = ld4g(phi + id + xs), PXM = ld4g(phi + id - xs);
  const float4 VP = ld4g(v + id + ys), V = ld4g(v + id), PYP = ld4g(phi + id + ys), PYM = ld4g(phi + id - ys);
  const float up[4] = {UP.x, UP.y, UP.z, UP.w}, uu[4] = {U.x, U.y, U.z, U.w};
  const float pxp[4] = {PXP.x, PXP.y, PXP.z, PXP.w}, pxm[4] = {PXM.x, PXM.y, PXM.z, PXM.w};
  const float vp[4] = {VP.x, VP.y, VP.z, VP.w}, vv[4] = {V.x, V.y, V.z, V.w};
  const float pyp[4] = {PYP.x, PYP.y, PYP.z, PYP.w}, pym[4] = {PYM.x, PYM.y, PYM.z, PYM.w};
  float o[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const float p = P.v[e + 1];
    const float du = up[e] * interp<float, IT>(up[e], p, pxp[e]) - uu[e] * interp<float, IT>(uu[e], pxm[e], p);
    const float dv = vp[e] * interp<float, IT>(vp[e], p, pyp[e]) - vv[e] * interp<float, IT>(vv[e], pym[e], p);
    const float wpk = W.v[e + 2], wij = W.v[e + 1];
    const float dw = wpk * interp<float, IT>(wpk, p, P.v[e + 2]) - wij * interp<float, IT>(wij, P.v[e], p);
    o[e] = (-du * ihx) - (dv * ihy) - (dw * ihz);
  }
  st4g(dphidt + id, o[0], o[1], o[2], o[3]);
  V4_END
}

// Self-advection on groups of four cells along k: the 17 rows it reads (u, v, w at the cell and
// its face neighbours) as 16-byte loads, the k-shifted values from the adjacent lanes; each
// component's expression is the scalar kernel's, in its order.
#ifndef OCU_ADVECT_SELF_MINB
#define OCU_ADVECT_SELF_MINB 2
#endif
// Neighbourhood of four cells k..k+3 of row (i, j) for the self-advection: rows with their
// k - 1 / k + 4 cells (Row4) and plain groups (float4); the suffixes give the (i, j) offsets
// (0, p = +1, m = -1).
struct SelfNbr {
  Row4 U00, Up0, V00, V0p, W00, Wm0, W0m;
  float4 Um0, U0p, U0m, Upm, Vm0, Vp0, V0m, Vmp, Wp0, W0p;
};

// The advection terms of u, v and w on the four cells (sol_selfadvection3ddev.cu:135-337 per
// cell, in its operand order), shared by the group kernel and the TMA-fed kernel.
template <int IT>
__device__ __forceinline__ void advect_self_group(const SelfNbr &n, float ihx, float ihy, float ihz, float ou[4],
                                                  float ov[4], float ow[4]) {
  const Row4 &U00 = n.U00, &Up0 = n.Up0, &V00 = n.V00, &V0p = n.V0p, &W00 = n.W00, &Wm0 = n.Wm0, &W0m = n.W0m;
  const float um0[4] = {n.Um0.x, n.Um0.y, n.Um0.z, n.Um0.w}, u0p[4] = {n.U0p.x, n.U0p.y, n.U0p.z, n.U0p.w};
  const float u0m[4] = {n.U0m.x, n.U0m.y, n.U0m.z, n.U0m.w}, upm[4] = {n.Upm.x, n.Upm.y, n.Upm.z, n.Upm.w};
  const float vm0[4] = {n.Vm0.x, n.Vm0.y, n.Vm0.z, n.Vm0.w}, vp0[4] = {n.Vp0.x, n.Vp0.y, n.Vp0.z, n.Vp0.w};
  const float v0m[4] = {n.V0m.x, n.V0m.y, n.V0m.z, n.V0m.w}, vmp[4] = {n.Vmp.x, n.Vmp.y, n.Vmp.z, n.Vmp.w};
  const float wp0[4] = {n.Wp0.x, n.Wp0.y, n.Wp0.z, n.Wp0.w}, w0p[4] = {n.W0p.x, n.W0p.y, n.W0p.z, n.W0p.w};
  const float half = 0.5f;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    // cell k = 4 k4 + e: Row4 index e + 1 is k, e + 2 is k + 1, e is k - 1
    const float ui = U00.v[e + 1], vi = V00.v[e + 1], wi = W00.v[e + 1];
    const float u_pi = Up0.v[e + 1], u_mi = um0[e], u_pj = u0p[e], u_mj = u0m[e], u_pk = U00.v[e + 2],
                u_mk = U00.v[e];
    const float v_pi = vp0[e], v_mi = vm0[e], v_pj = V0p.v[e + 1], v_mj = v0m[e], v_pk = V00.v[e + 2],
                v_mk = V00.v[e];
    const float w_pi = wp0[e], w_mi = Wm0.v[e + 1], w_pj = w0p[e], w_mj = W0m.v[e + 1], w_pk = W00.v[e + 2],
                w_mk = W00.v[e];
    float a, b, d1, d2, d3;
    a = half * (ui + u_pi);
    b = half * (ui + u_mi);
    d1 = (a * interp<float, IT>(a, ui, u_pi)) - (b * interp<float, IT>(b, u_mi, ui));
    a = half * (v_pj + vmp[e]);
    b = half * (vi + v_mi);
    d2 = (a * interp<float, IT>(a, ui, u_pj)) - (b * interp<float, IT>(b, u_mj, ui));
    a = half * (w_pk + Wm0.v[e + 2]);
    b = half * (wi + w_mi);
    d3 = (a * interp<float, IT>(a, ui, u_pk)) - (b * interp<float, IT>(b, u_mk, ui));
    ou[e] = -d1 * ihx - d2 * ihy - d3 * ihz;

    a = half * (u_pi + upm[e]);
    b = half * (ui + u_mj);
    d1 = (a * interp<float, IT>(a, vi, v_pi)) - (b * interp<float, IT>(b, v_mi, vi));
    a = half * (vi + v_pj);
    b = half * (vi + v_mj);
    d2 = (a * interp<float, IT>(a, vi, v_pj)) - (b * interp<float, IT>(b, v_mj, vi));
    a = half * (w_pk + W0m.v[e + 2]);
    b = half * (wi + w_mj);
    d3 = (a * interp<float, IT>(a, vi, v_pk)) - (b * interp<float, IT>(b, v_mk, vi));
    ov[e] = -d1 * ihx - d2 * ihy - d3 * ihz;

    a = half * (u_pi + Up0.v[e]);
    b = half * (ui + u_mk);
    d1 = (a * interp<float, IT>(a, wi, w_pi)) - (b * interp<float, IT>(b, w_mi, wi));
    a = half * (v_pj + V0p.v[e]);
    b = half * (vi + v_mk);
    d2 = (a * interp<float, IT>(a, wi, w_pj)) - (b * interp<float, IT>(b, w_mj, wi));
    a = half * (wi + w_pk);
    b = half * (wi + w_mk);
    d3 = (a * interp<float, IT>(a, wi, w_pk)) - (b * interp<float, IT>(b, w_mk, wi));
    ow[e] = -d1 * ihx - d2 * ihy - d3 * ihz;
  }
}

template <int IT>
__global__ void __launch_bounds__(256, OCU_ADVECT_SELF_MINB) k_advect_self_v4(const float *__restrict__ u, const float *__restrict__ v,
                                                           const float *__restrict__ w, float *__restrict__ dudt,
                                                           float *__restrict__ dvdt, float *__restrict__ dwdt, float ihx,
                                                           float ihy, float ihz, long long xs, long long ys, int nx,
                                                           int ny, int nz4) {
  V4_BEGIN
  // rows with their k - 1 / k + 4 neighbours (every lane takes part in the shuffles)
  SelfNbr n;
  n.U00 = row4(u, id, ok, first, last);
  n.Up0 = row4(u, id + xs, ok, first, last);
  n.V00 = row4(v, id, ok, first, last);
  n.V0p = row4(v, id + ys, ok, first, last);
  n.W00 = row4(w, id, ok, first, last);
  n.Wm0 = row4(w, id - xs, ok, first, last);
  n.W0m = row4(w, id - ys, ok, first, last);
  if (!ok) continue;
  n.Um0 = ld4g(u + id - xs); n.U0p = ld4g(u + id + ys); n.U0m = ld4g(u + id - ys); n.Upm = ld4g(u + id + xs - ys);
  n.Vm0 = ld4g(v + id - xs); n.Vp0 = ld4g(v + id + xs); n.V0m = ld4g(v + id - ys); n.Vmp = ld4g(v + id - xs + ys);
  n.Wp0 = ld4g(w + id + xs); n.W0p = ld4g(w + id + ys);
  float ou[4], ov[4], ow[4];
  advect_self_group<IT>(n, ihx, ihy, ihz, ou, ov, ow);
  st4g(dudt + id, ou[0], ou[1], ou[2], ou[3]);
  st4g(dvdt + id, ov[0], ov[1], ov[2], ov[3]);
  st4g(dwdt + id, ow[0], ow[1], ow[2], ow[3]);
  V4_END
}

// whether the FP32 group form applies: nz, the strides and every array's interior origin on
// 16-byte boundaries
static bool v4_ok(int nz, const ocu_layout &L, std::initializer_list<const void *> origins) {
  if (nz % 4 || L.xstride % 4 || L.ystride % 4) return false;
  for (const void *p : origins)
    if (reinterpret_cast<uintptr_t>(p) % 16) return false;
  return true;
}

// Blocks of 256 threads, whole warps: a block row is the row's nz/4 groups when that divides 32
// (a warp then holds several rows), else 32 (lanes past the row's end idle).  Every lane of a
// warp takes part in the shuffles.
static inline void shape_v4(int nx, int ny, int nz, dim3 *grid, dim3 *block, int ci = kCellsIV) {
  const int nz4 = nz / 4;
  const int bx = (nz4 < 32 && 32 % nz4 == 0) ? nz4 : 32;
  *block = dim3(bx, 256 / bx);
  *grid = dim3((nz4 + bx - 1) / bx, (ny + block->y - 1) / block->y, (nx + ci - 1) / ci);
}

template <typename T>
ocu_status launch_divergence(const T *u, const T *v, const T *w, T *div, const ocu_layout &L,
                             int nx, int ny, int nz, double hx, double hy, double hz,
                             cudaStream_t s) {
  dim3 g, b;
  if constexpr (sizeof(T) == 4) {
    if (v4_ok(nz, L, {u, v, w, div})) {
      shape_v4(nx, ny, nz, &g, &b);
      k_divergence_v4<<<g, b, 0, s>>>(u, v, w, div, (T)(1 / hx), (T)(1 / hy), (T)(1 / hz), L.xstride, L.ystride, nx,
                                      ny, nz / 4);
      return check_launch("k_divergence_v4");
    }
  }
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
  if constexpr (sizeof(T) == 4) {
    if (v4_ok(nz, L, {u, v, w, phi})) {
      shape_v4(nx, ny, nz, &g, &b);
      k_gradient_v4<<<g, b, 0, s>>>(u, v, w, phi, coefficient, (T)(1 / hx), (T)(1 / hy), (T)(1 / hz), L.xstride,
                                    L.ystride, nx, ny, nz / 4);
      return check_launch("k_gradient_v4");
    }
  }
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
  if constexpr (sizeof(T) == 4) {
    const int nz4 = nz / 4, nr = nz - 4 * nz4;
    if (nz4 > 0 && v4_ok(4 * nz4, L, {phi, dphidt})) {
      const T ihx2 = (T)(1 / (hx * hx)), ihy2 = (T)(1 / (hy * hy)), ihz2 = (T)(1 / (hz * hz));
      shape_v4(nx, ny, 4 * nz4, &g, &b);
      k_laplacian_v4<false><<<g, b, 0, s>>>(phi, dphidt, ihx2, ihy2, ihz2, coefficient, L.xstride, L.ystride, nx, ny,
                                            nz4, nr, ThermalArgs{});
      return check_launch("k_laplacian_v4");
    }
  }
  shape(nx, ny, nz, &g, &b);
  k_laplacian<T><<<g, b, 0, s>>>(phi, dphidt, (T)(1 / (hx * hx)), (T)(1 / (hy * hy)), (T)(1 / (hz * hz)),
                                 coefficient, L.xstride, L.ystride, nx, ny, nz);
  return check_launch("k_laplacian");
}

// The diffusion of the vertical velocity component and its buoyancy in one pass (FP32 group
// form only); OCU_ERR_UNSUPPORTED when it does not apply, and the caller launches the two.
ocu_status launch_laplacian_thermal(const float *phi, float *dphidt, const ocu_layout &L, int nx, int ny, int nz,
                                    double hx, double hy, double hz, float coefficient, const float *temp, float ct,
                                    long long nbr, int tnx, int tny, int tnz, cudaStream_t s) {
  const int nz4 = nz / 4, nr = nz - 4 * nz4;
  // the temperature is read at the velocity's index (one layout), and its vertical neighbour one
  // cell down (from the lanes) or a whole group away
  if (nz4 == 0 || (nbr != 1 && nbr % 4 != 0) || !v4_ok(4 * nz4, L, {phi, dphidt, temp})) return OCU_ERR_UNSUPPORTED;
  dim3 g, b;
  shape_v4(nx, ny, 4 * nz4, &g, &b);
  k_laplacian_v4<true><<<g, b, 0, s>>>(phi, dphidt, (float)(1 / (hx * hx)), (float)(1 / (hy * hy)),
                                       (float)(1 / (hz * hz)), coefficient, L.xstride, L.ystride, nx, ny, nz4, nr,
                                       ThermalArgs{temp, ct, nbr, tnx, tny, tnz});
  return check_launch("k_laplacian_v4");
}

template <typename T>
ocu_status launch_advect_self(const T *u, const T *v, const T *w, T *du, T *dv, T *dw,
                              const ocu_layout &L, int nx, int ny, int nz, double hx, double hy,
                              double hz, int it, cudaStream_t s) {
  dim3 g, b;
  const T ihx = (T)(1 / hx), ihy = (T)(1 / hy), ihz = (T)(1 / hz);
  if constexpr (sizeof(T) == 4) {
    if ((it == OCU_IT_FIRST_ORDER_UPWIND || it == OCU_IT_SECOND_ORDER_CENTERED) && v4_ok(nz, L, {u, v, w, du, dv, dw})) {
      shape_v4(nx, ny, nz, &g, &b);
      if (it == OCU_IT_FIRST_ORDER_UPWIND)
        k_advect_self_v4<OCU_IT_FIRST_ORDER_UPWIND><<<g, b, 0, s>>>(u, v, w, du, dv, dw, ihx, ihy, ihz, L.xstride,
                                                                   L.ystride, nx, ny, nz / 4);
      else
        k_advect_self_v4<OCU_IT_SECOND_ORDER_CENTERED><<<g, b, 0, s>>>(u, v, w, du, dv, dw, ihx, ihy, ihz,
                                                                      L.xstride, L.ystride, nx, ny, nz / 4);
      return check_launch("k_advect_self_v4");
    }
  }
  shape(nx, ny, nz, &g, &b, 1);
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

// ---- self-advection fed by TMA ----------------------------------------------------------------
// A CTA owns a (j, k) tile -- TY rows of TZ cells -- and marches along i over a run of planes.
// Each plane of u, v and w over the tile with a one-row halo in j and a 16-byte halo in k comes
// into shared memory by one 3-D TMA box load per field (cp.async.bulk.tensor, mbarrier
// completion), issued by one thread three planes ahead of its use; a thread then computes four
// cells of the tile's plane i from planes i-1, i and i+1 in shared memory and stores the three
// results as 16-byte writes.  Every operand is the group kernel's (advect_self_group), so the
// results are bit-identical to it.  Work split: the (tile, plane) steps of the grid are cut
// into equal contiguous ranges, one per resident CTA (tile-major: a range is one or two runs of
// planes), so a tile's halo planes are loaded twice per run only.
#ifndef OCU_ADV_TMA_NS
#define OCU_ADV_TMA_NS 4
#endif
#ifndef OCU_ADV_TMA_MINB
#define OCU_ADV_TMA_MINB 3
#endif
template <int TZ>
struct AdvTile {
  static constexpr int BX = TZ / 4;                        // threads along k (a float4 group each)
  static constexpr int TY = 256 / BX;                      // rows (j)
  static constexpr int H = 4;                              // k halo: one 16-byte granule
  static constexpr int W = TZ + 2 * H;                     // shared row pitch (floats)
  static constexpr int R = TY + 2;                         // rows j0-1 .. j0+TY
  static constexpr int PLANE = (W * R + 31) / 32 * 32;     // floats, a multiple of 128 bytes
  static constexpr int NS = OCU_ADV_TMA_NS;                // buffers per field: i-1, i, i+1, the rest ahead
  static constexpr int THREADS = 256;
  // plane buffers, NS mbarriers, the abort word (8 bytes), the barrier of the timeout test
  // (8 bytes); +128 to align the base by hand
  static constexpr size_t SMEM = (size_t)3 * NS * PLANE * sizeof(float) + NS * 8 + 16 + 128;
};

struct AdvArgs {
  long long xs, ys;   // strides of the interior-origin pointers (elements)
  int nx, ny, nz;
  int gx, gy;         // ghost widths (view coordinates)
  int ntz;            // tiles along k
  long long steps;    // tiles * nx
  int wait_limit;     // polls of a load wait before the launch gives up
  int stall_test;     // testing the timeout path: the first wait is on a barrier nothing completes
};

template <int TZ, int IT>
__global__ void __launch_bounds__(256, OCU_ADV_TMA_MINB) k_advect_self_tma(
    const __grid_constant__ CUtensorMap tm_u, const __grid_constant__ CUtensorMap tm_v,
    const __grid_constant__ CUtensorMap tm_w, float *__restrict__ dudt, float *__restrict__ dvdt,
    float *__restrict__ dwdt, float ihx, float ihy, float ihz, AdvArgs a, int *__restrict__ err) {
  using S = AdvTile<TZ>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA destinations must be 128-byte aligned: align the base explicitly
  float *sm = reinterpret_cast<float *>(smem_raw + ((128 - (smem_addr(smem_raw) & 127)) & 127));
  constexpr int FIELD = S::NS * S::PLANE;  // field f's buffers start at sm + f * FIELD
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm + 3 * FIELD);
  int &abort_flag = *reinterpret_cast<int *>(bar + S::NS);
  unsigned long long *stall_bar = bar + S::NS + 1;  // never arrived at: only the timeout test waits on it

  const unsigned bytes = 3u * S::W * S::R * (unsigned)sizeof(float);
  const long long lo = a.steps * blockIdx.x / gridDim.x, hi = a.steps * (blockIdx.x + 1) / gridDim.x;
  const int tx = threadIdx.x % S::BX, ty = threadIdx.x / S::BX;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int q = 0; q < S::NS; q++) mbar_init(&bar[q], 1);
    mbar_init(stall_bar, 1);
    mbar_init_fence();
    tma_prefetch_map(&tm_u);
    tma_prefetch_map(&tm_v);
    tma_prefetch_map(&tm_w);
  }
  __syncthreads();
  if (a.stall_test) {
    // the timeout path without a fault: a wait that nothing completes runs out of polls before
    // any load is issued, so the CTA has nothing in flight when it returns
    if (threadIdx.x == 0 && !mbar_wait_bounded(stall_bar, 0u, a.wait_limit)) {
      atomicOr(err, 1);
      abort_flag = 1;
    }
    __syncthreads();
    if (abort_flag) return;
  }

  int gbase = 0;   // loads are numbered across this CTA's runs: buffer = g % NS
  int issued = 0;  // (thread 0) loads issued in the current run
  for (long long idx = lo; idx < hi;) {
    const int tile = (int)(idx / a.nx);
    const int ia = (int)(idx % a.nx);
    const int ib = (int)((long long)ia + (hi - idx) < a.nx ? ia + (hi - idx) : a.nx);
    idx += ib - ia;
    const int k0 = (tile % a.ntz) * TZ, j0 = (tile / a.ntz) * S::TY;
    const int nload = ib - ia + 2;  // planes ia-1 .. ib
    auto issue = [&](int m) {       // load m of this run: plane ia-1+m of u, v and w
      const int g = gbase + m;
      unsigned long long *bm = &bar[g % S::NS];
      float *dst = sm + (g % S::NS) * S::PLANE;
      const int pz = ia - 1 + m + a.gx, py = j0 - 1 + a.gy;
      mbar_expect_tx(bm, bytes);
      // view x = k + H: the box starts at k = k0 - H
      tma_load_3d(dst, &tm_u, k0, py, pz, bm);
      tma_load_3d(dst + FIELD, &tm_v, k0, py, pz, bm);
      tma_load_3d(dst + 2 * FIELD, &tm_w, k0, py, pz, bm);
    };
    // the previous run's buffers are no longer read; order those reads before the new loads
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0)
      for (issued = 0; issued < nload && issued < S::NS; issued++) issue(issued);

    for (int n = 0; n < ib - ia; n++) {
      const int s = ia + n;  // plane computed: loads n (plane s-1), n+1 (s), n+2 (s+1)
      if (threadIdx.x == 0) {
        for (int m = (n == 0 ? 0 : n + 2); m <= n + 2; m++) {
          const int g = gbase + m;
          if (!mbar_wait_bounded(&bar[g % S::NS], (unsigned)((g / S::NS) & 1), a.wait_limit)) {
            atomicOr(err, 1);
            abort_flag = 1;
            // let the copies already issued -- the one waited for included -- land before the
            // CTA's shared memory goes away (each wait again bounded, by the default limit)
            for (int q = m; q < issued; q++)
              mbar_wait_bounded(&bar[(gbase + q) % S::NS], (unsigned)(((gbase + q) / S::NS) & 1), kWaitLimit);
            break;
          }
        }
      }
      __syncthreads();
      if (abort_flag) return;
      const int g = gbase + n;
      const float *um = sm + (g % S::NS) * S::PLANE, *uc = sm + ((g + 1) % S::NS) * S::PLANE;
      const float *up = sm + ((g + 2) % S::NS) * S::PLANE;
      const float *vm = um + FIELD, *vc = uc + FIELD, *vp = up + FIELD;
      const float *wm = um + 2 * FIELD, *wc = uc + 2 * FIELD, *wp = up + 2 * FIELD;
      const int j = j0 + ty, k = k0 + 4 * tx;
      if (j < a.ny && k < a.nz) {
        const int r = ty + 1, cb = 4 * tx + S::H;
        // a row's group with its k - 1 / k + 4 cells (warp shuffles for these measured slower:
        // 61.6 against 55.9 us at 256x256x128)
        auto row6 = [&](const float *p, int rr) {
          const float *q = p + rr * S::W + cb;
          const float4 c = *reinterpret_cast<const float4 *>(q);
          Row4 o;
          o.v[0] = q[-1]; o.v[1] = c.x; o.v[2] = c.y; o.v[3] = c.z; o.v[4] = c.w; o.v[5] = q[4];
          return o;
        };
        auto grp = [&](const float *p, int rr) { return *reinterpret_cast<const float4 *>(p + rr * S::W + cb); };
        SelfNbr nb;
        nb.U00 = row6(uc, r); nb.Up0 = row6(up, r);
        nb.V00 = row6(vc, r); nb.V0p = row6(vc, r + 1);
        nb.W00 = row6(wc, r); nb.Wm0 = row6(wm, r); nb.W0m = row6(wc, r - 1);
        nb.Um0 = grp(um, r); nb.U0p = grp(uc, r + 1); nb.U0m = grp(uc, r - 1); nb.Upm = grp(up, r - 1);
        nb.Vm0 = grp(vm, r); nb.Vp0 = grp(vp, r); nb.V0m = grp(vc, r - 1); nb.Vmp = grp(vm, r + 1);
        nb.Wp0 = grp(wp, r); nb.W0p = grp(wc, r + 1);
        float ou[4], ov[4], ow[4];
        advect_self_group<IT>(nb, ihx, ihy, ihz, ou, ov, ow);
        const long long id = (long long)s * a.xs + (long long)j * a.ys + k;
        st4g(dudt + id, ou[0], ou[1], ou[2], ou[3]);
        st4g(dvdt + id, ov[0], ov[1], ov[2], ov[3]);
        st4g(dwdt + id, ow[0], ow[1], ow[2], ow[3]);
      }
      // every thread is done with plane s-1's buffers: the next load reuses them
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (threadIdx.x == 0 && issued < nload) issue(issued++);
    }
    gbase += nload;
  }
}

// View of a field for the TMA loads: x = k + H (base = row (i=-gx, j=-gy) at k = -H, which is
// pre-padding of that row), dims {nz+H+1, pny, pnx}: both z ghosts inside, and the view's last
// element inside the allocation (pnz >= nz + H + 1); box = one plane of a tile with its halos.
template <int TZ>
static ocu_status make_adv_tmap(const float *origin_ptr, const ocu_layout &L, CUtensorMap *out) {
  using S = AdvTile<TZ>;
  auto fn = encode_fn();
  if (!fn) return fail(OCU_ERR_CUDA, "[ERROR] cuTensorMapEncodeTiled is not available");
  const float *base = origin_ptr - (long long)L.gx * L.xstride - (long long)L.gy * L.ystride - S::H;
  cuuint64_t dims[3] = {(cuuint64_t)(L.nz + S::H + 1), (cuuint64_t)L.pny, (cuuint64_t)L.pnx};
  cuuint64_t strides[2] = {(cuuint64_t)L.ystride * sizeof(float), (cuuint64_t)L.xstride * sizeof(float)};
  cuuint32_t box[3] = {(cuuint32_t)S::W, (cuuint32_t)S::R, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(OCU_ERR_CUDA, "[ERROR] cuTensorMapEncodeTiled failed (%d)", (int)r);
  return OCU_OK;
}

// Resident CTAs of the TMA kernel per device, computed once per (device, tile width).
template <int TZ, int IT>
static ocu_status adv_slots(int *slots) {
  using S = AdvTile<TZ>;
  static int cache[64] = {0};
  static std::mutex mu;
  int dev = 0;
  OCU_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
  std::lock_guard<std::mutex> lock(mu);
  if (!cache[dev & 63]) {
    OCU_TRY(check_cuda(cudaFuncSetAttribute(k_advect_self_tma<TZ, IT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)S::SMEM),
                       "cudaFuncSetAttribute (advection)"));
    int per_sm = 0, sms = 0;
    OCU_TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_advect_self_tma<TZ, IT>, S::THREADS,
                                                                     S::SMEM),
                       "cudaOccupancyMaxActiveBlocksPerMultiprocessor"));
    OCU_TRY(check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute"));
    cache[dev & 63] = per_sm * sms > 0 ? per_sm * sms : 1;
  }
  *slots = cache[dev & 63];
  return OCU_OK;
}

// OCU_B200_ADVECT_TMA=0 never takes the TMA form, =1 takes it wherever it applies (for tests);
// unset: where every CTA gets at least kAdvTmaMinSteps planes (below that the halo planes
// cost more than they save, and the grid's fields fit in L2 anyway).
constexpr long long kAdvTmaMinSteps = 16;

template <int TZ, int IT>
static ocu_status launch_adv_tma_t(const float *u, const float *v, const float *w, float *du, float *dv, float *dw,
                                   const ocu_layout &L, int nx, int ny, int nz, float ihx, float ihy, float ihz,
                                   int force, int *err, int wait_limit, cudaStream_t s) {
  using S = AdvTile<TZ>;
  AdvArgs a;
  a.xs = L.xstride; a.ys = L.ystride;
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.gx = L.gx; a.gy = L.gy;
  a.ntz = (nz + TZ - 1) / TZ;
  a.steps = (long long)a.ntz * ((ny + S::TY - 1) / S::TY) * nx;
  a.stall_test = wait_limit < 0;
  a.wait_limit = wait_limit < 0 ? -wait_limit : (wait_limit > 0 ? wait_limit : kWaitLimit);
  int slots = 1;
  OCU_TRY((adv_slots<TZ, IT>(&slots)));
  if (!force && a.steps < kAdvTmaMinSteps * slots) return OCU_ERR_UNSUPPORTED;
  const long long grid = a.steps < slots ? a.steps : slots;
  CUtensorMap tu, tv, tw;
  OCU_TRY(make_adv_tmap<TZ>(u, L, &tu));
  OCU_TRY(make_adv_tmap<TZ>(v, L, &tv));
  OCU_TRY(make_adv_tmap<TZ>(w, L, &tw));
  k_advect_self_tma<TZ, IT><<<(unsigned)grid, S::THREADS, S::SMEM, s>>>(tu, tv, tw, du, dv, dw, ihx, ihy, ihz, a, err);
  return check_launch("k_advect_self_tma");
}

ocu_status launch_advect_self_tma(const float *u, const float *v, const float *w, float *du, float *dv, float *dw,
                                  const ocu_layout &L, int nx, int ny, int nz, double hx, double hy, double hz,
                                  int it, int *err, int wait_limit, cudaStream_t s) {
  const char *e = std::getenv("OCU_B200_ADVECT_TMA");
  const int mode = e ? std::atoi(e) : -1;
  if (mode == 0 || !err) return OCU_ERR_UNSUPPORTED;
  if (it != OCU_IT_FIRST_ORDER_UPWIND && it != OCU_IT_SECOND_ORDER_CENTERED) return OCU_ERR_UNSUPPORTED;
  // one ghost layer on every side, 16-byte groups along k, and the view's conditions
  if (L.gx != 1 || L.gy != 1 || L.gz != 1 || nz % 4 || nz < 32 || L.pnz < nz + AdvTile<32>::H + 1) return OCU_ERR_UNSUPPORTED;
  if (!v4_ok(nz, L, {u, v, w, du, dv, dw})) return OCU_ERR_UNSUPPORTED;
  const float ihx = (float)(1 / hx), ihy = (float)(1 / hy), ihz = (float)(1 / hz);
  const int force = mode == 1;
  if (it == OCU_IT_FIRST_ORDER_UPWIND) {
    if (nz >= 128)
      return launch_adv_tma_t<128, OCU_IT_FIRST_ORDER_UPWIND>(u, v, w, du, dv, dw, L, nx, ny, nz, ihx, ihy, ihz, force,
                                                              err, wait_limit, s);
    if (nz >= 64)
      return launch_adv_tma_t<64, OCU_IT_FIRST_ORDER_UPWIND>(u, v, w, du, dv, dw, L, nx, ny, nz, ihx, ihy, ihz, force,
                                                             err, wait_limit, s);
    return launch_adv_tma_t<32, OCU_IT_FIRST_ORDER_UPWIND>(u, v, w, du, dv, dw, L, nx, ny, nz, ihx, ihy, ihz, force,
                                                           err, wait_limit, s);
  }
  if (nz >= 128)
    return launch_adv_tma_t<128, OCU_IT_SECOND_ORDER_CENTERED>(u, v, w, du, dv, dw, L, nx, ny, nz, ihx, ihy, ihz,
                                                               force, err, wait_limit, s);
  if (nz >= 64)
    return launch_adv_tma_t<64, OCU_IT_SECOND_ORDER_CENTERED>(u, v, w, du, dv, dw, L, nx, ny, nz, ihx, ihy, ihz,
                                                              force, err, wait_limit, s);
  return launch_adv_tma_t<32, OCU_IT_SECOND_ORDER_CENTERED>(u, v, w, du, dv, dw, L, nx, ny, nz, ihx, ihy, ihz, force,
                                                            err, wait_limit, s);
}

template <typename T>
ocu_status launch_advect_passive(const T *u, const T *v, const T *w, const T *phi, T *dphi,
                                 const ocu_layout &L, int nx, int ny, int nz, double hx,
                                 double hy, double hz, int it, cudaStream_t s) {
  dim3 g, b;
  const T ihx = (T)(1 / hx), ihy = (T)(1 / hy), ihz = (T)(1 / hz);
  if constexpr (sizeof(T) == 4) {
    if ((it == OCU_IT_FIRST_ORDER_UPWIND || it == OCU_IT_SECOND_ORDER_CENTERED) && v4_ok(nz, L, {u, v, w, phi, dphi})) {
      shape_v4(nx, ny, nz, &g, &b, kCellsIPassive);
      if (it == OCU_IT_FIRST_ORDER_UPWIND)
        k_advect_passive_v4<OCU_IT_FIRST_ORDER_UPWIND><<<g, b, 0, s>>>(u, v, w, phi, dphi, ihx, ihy, ihz, L.xstride,
                                                                      L.ystride, nx, ny, nz / 4);
      else
        k_advect_passive_v4<OCU_IT_SECOND_ORDER_CENTERED><<<g, b, 0, s>>>(u, v, w, phi, dphi, ihx, ihy, ihz,
                                                                         L.xstride, L.ystride, nx, ny, nz / 4);
      return check_launch("k_advect_passive_v4");
    }
  }
  shape(nx, ny, nz, &g, &b);
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
  if constexpr (sizeof(T) == 4) {
    if ((nbr_stride == 1 || nbr_stride % 4 == 0) && v4_ok(nz, L, {dvdt, temp})) {
      shape_v4(nx, ny, nz, &g, &b);
      k_thermal_force_v4<<<g, b, 0, s>>>(dvdt, coefficient, temp, nbr_stride, L.xstride, L.ystride, nx, ny, nz / 4);
      return check_launch("k_thermal_force_v4");
    }
  }
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
