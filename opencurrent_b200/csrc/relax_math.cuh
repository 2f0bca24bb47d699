// Per-cell red-black SOR arithmetic shared by every relax kernel (one definition, so the
// in-place colour sweeps, the two-colour shared-memory pass and the coarse tail agree bit for
// bit).
#pragma once

#include "mg_fused.h"

namespace ocub {

// One red-black SOR update from the cell's value, its right-hand side and its six neighbours
// (z-, z+, y-, y+, x-, x+); arithmetic of the reference's colour kernels
// (sol_mgpressure3ddev.cu:145-230): residual sequence, boundary-aware diagonal, then
// u + omega * res / diag.
template <typename T>
__device__ __forceinline__ T relax_res(T uc, T bv, T zm, T zp, T ym, T yp, T xm, T xp, const RelaxCoefD<T> &c) {
  T res;
  if (sizeof(T) == 4) {
    res = (-c.hsq * bv - c.ld * uc);
    res += c.fz * (zm + zp);
    res += c.fy * (ym + yp);
    res += c.fx * (xm + xp);
  } else {
    res = -c.ld * uc;
    res += c.fz * (zm + zp);
    res += c.fy * (ym + yp);
    res += c.fx * (xm + xp);
    res += c.hsq * bv;
  }
  return res;
}

// Diagonal of cell (i,j,k); away from every face it is c.ld exactly (nothing is added).
template <typename T>
__device__ __forceinline__ T relax_dg(int i, int j, int k, int nx, int ny, int nz, const RelaxCoefD<T> &c,
                                      const T *__restrict__ diag) {
  T dg;
  if (sizeof(T) == 4 || !diag) {  // FP64: same sequence the 2D table is built with (sol_mgpressure3ddev.cu:36-41)
    dg = c.ld;
    if (i == nx - 1) dg += c.xp;
    if (i == 0) dg += c.xn;
    if (j == ny - 1) dg += c.yp;
    if (j == 0) dg += c.yn;
  } else {
    dg = diag[(long long)i * ny + j];
  }
  if (k == nz - 1) dg += c.zp;
  if (k == 0) dg += c.zn;
  return dg;
}

template <typename T>
__device__ __forceinline__ T relax_value(T uc, T bv, T zm, T zp, T ym, T yp, T xm, T xp, int i, int j, int k,
                                         int nx, int ny, int nz, const RelaxCoefD<T> &c,
                                         const T *__restrict__ diag) {
  const T res = relax_res<T>(uc, bv, zm, zp, ym, yp, xm, xp, c);
  const T dg = relax_dg<T>(i, j, k, nx, ny, nz, c, diag);
  return uc + c.omega * res / dg;
}

template <typename T>
__device__ __forceinline__ T relax_point(const T *__restrict__ u, const T *__restrict__ b, long long id, long long xs,
                                         long long ys, int i, int j, int k, int nx, int ny, int nz,
                                         const RelaxCoefD<T> &c, const T *__restrict__ diag) {
  return relax_value<T>(u[id], b[id], u[id - 1], u[id + 1], u[id - ys], u[id + ys], u[id - xs], u[id + xs], i, j, k,
                        nx, ny, nz, c, diag);
}

// Residual b - L u of one cell (devf.cu:68-90, devd.cu:94-114), the operand order of every
// residual kernel.
template <typename T>
__device__ __forceinline__ T residual_at(const T *__restrict__ u, const T *__restrict__ b, long long id, long long xs,
                                         long long ys, const ResCoefT<T> &c) {
  return b[id] - (c.fzh * (u[id - 1] + u[id + 1]) + c.fyh * (u[id - ys] + u[id + ys]) +
                  c.fxh * (u[id - xs] + u[id + xs]) - c.dg * u[id]);
}

}  // namespace ocub
