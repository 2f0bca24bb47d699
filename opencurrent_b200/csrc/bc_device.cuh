// Device-side ghost-cell rules shared by the grid and multigrid kernels.
#pragma once

#include "ocu_internal.h"

namespace ocub {

enum { FX_POS = 0, FX_NEG = 1, FY_POS = 2, FY_NEG = 3, FZ_POS = 4, FZ_NEG = 5 };

// ------------------------------------------------------------------------------------------
// Scalar ghost fill, level1 (faces + edges + corners) in ONE launch.
//
// The reference fills x faces, then y faces over i in [-1,nx] (reading the x ghosts), then z
// faces over i in [-1,nx], j in [-1,ny] (grid3dboundary.cu:237-347, 756-820).  Every ghost value
// is therefore a composition of the face rules applied to one interior cell.  Each thread here
// owns one ghost cell, evaluates that composition from interior values only, and writes it;
// faces of type BC_NONE are never written (their stale value is what the reference reads
// back).  Dirichlet: -src + 2*value (2*value in float); Neumann: src -/+ h*value, in T.
// ------------------------------------------------------------------------------------------
template <typename T>
struct Level1Compose {
  T *p;
  long long xs, ys;
  int nx, ny, nz;
  BCDev bc;
  T hx, hy, hz;

  __device__ __forceinline__ T mem(int i, int j, int k) const {
    return p[(long long)i * xs + (long long)j * ys + k];
  }
  __device__ __forceinline__ static bool writes(int t) {
    return t == OCU_BC_PERIODIC || t == OCU_BC_DIRICHELET || t == OCU_BC_NEUMANN;
  }
  __device__ __forceinline__ static T dir(T src, float v) { return -src + (T)(2 * v); }

  // value after the x pass; j, k interior
  __device__ T ax(int i, int j, int k) const {
    if (i >= 0 && i < nx) return mem(i, j, k);
    const bool neg = i < 0;
    const int f = neg ? FX_NEG : FX_POS;
    const int t = bc.ty(f);
    const float v = bc.val(f);
    if (t == OCU_BC_PERIODIC) return mem(neg ? nx - 1 : 0, j, k);
    if (t == OCU_BC_DIRICHELET) return dir(mem(neg ? 0 : nx - 1, j, k), v);
    if (t == OCU_BC_NEUMANN) return neg ? mem(0, j, k) - hx * (T)v : mem(nx - 1, j, k) + hx * (T)v;
    return mem(i, j, k);
  }
  // value after the y pass; k interior, i in [-1,nx]
  __device__ T ay(int i, int j, int k) const {
    if (j >= 0 && j < ny) return ax(i, j, k);
    const bool neg = j < 0;
    const int f = neg ? FY_NEG : FY_POS;
    const int t = bc.ty(f);
    const float v = bc.val(f);
    if (t == OCU_BC_PERIODIC) return ax(i, neg ? ny - 1 : 0, k);
    if (t == OCU_BC_DIRICHELET) return dir(ax(i, neg ? 0 : ny - 1, k), v);
    if (t == OCU_BC_NEUMANN) return neg ? ax(i, 0, k) - hy * (T)v : ax(i, ny - 1, k) + hy * (T)v;
    return mem(i, j, k);
  }
  // value after the z pass; i in [-1,nx], j in [-1,ny]
  __device__ T az(int i, int j, int k) const {
    if (k >= 0 && k < nz) return ay(i, j, k);
    const bool neg = k < 0;
    const int f = neg ? FZ_NEG : FZ_POS;
    const int t = bc.ty(f);
    const float v = bc.val(f);
    if (t == OCU_BC_PERIODIC) return ay(i, j, neg ? nz - 1 : 0);
    if (t == OCU_BC_DIRICHELET) return dir(ay(i, j, neg ? 0 : nz - 1), v);
    if (t == OCU_BC_NEUMANN) return neg ? ay(i, j, 0) - hz * (T)v : ay(i, j, nz - 1) + hz * (T)v;
    return mem(i, j, k);
  }
};

// The whole level1 fill executed by one thread block (the composition reads interior values
// only, so every ghost can be written in the same phase).
template <typename T>
__device__ void level1_fill_block(T *u, long long xs, long long ys, int nx, int ny, int nz, const BCDev &bc, T hx,
                                  T hy, T hz) {
  Level1Compose<T> lc;
  lc.p = u; lc.xs = xs; lc.ys = ys; lc.nx = nx; lc.ny = ny; lc.nz = nz; lc.bc = bc;
  lc.hx = hx; lc.hy = hy; lc.hz = hz;
  const int zr = 2 * (nx + 2) * (ny + 2), yr = 2 * (nx + 2) * nz, xr = 2 * ny * nz;
  for (int q = threadIdx.x; q < zr + yr + xr; q += blockDim.x) {
    int r = q;
    if (r < zr) {
      const int per = (nx + 2) * (ny + 2), side = r / per, i = (r % per) / (ny + 2) - 1, j = (r % per) % (ny + 2) - 1;
      if (Level1Compose<T>::writes(bc.ty(side ? FZ_POS : FZ_NEG)))
        u[(long long)i * xs + (long long)j * ys + (side ? nz : -1)] = lc.az(i, j, side ? nz : -1);
      continue;
    }
    r -= zr;
    if (r < yr) {
      const int per = (nx + 2) * nz, side = r / per, i = (r % per) / nz - 1, k = (r % per) % nz;
      if (Level1Compose<T>::writes(bc.ty(side ? FY_POS : FY_NEG)))
        u[(long long)i * xs + (long long)(side ? ny : -1) * ys + k] = lc.ay(i, side ? ny : -1, k);
      continue;
    }
    r -= yr;
    {
      const int per = ny * nz, side = r / per, j = (r % per) / nz, k = (r % per) % nz;
      if (Level1Compose<T>::writes(bc.ty(side ? FX_POS : FX_NEG)))
        u[(long long)(side ? nx : -1) * xs + (long long)j * ys + k] = lc.ax(side ? nx : -1, j, k);
    }
  }
}

}  // namespace ocub
