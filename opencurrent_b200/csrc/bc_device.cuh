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
    const int t = bc.type[f];
    const float v = bc.value[f];
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
    const int t = bc.type[f];
    const float v = bc.value[f];
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
    const int t = bc.type[f];
    const float v = bc.value[f];
    if (t == OCU_BC_PERIODIC) return ay(i, j, neg ? nz - 1 : 0);
    if (t == OCU_BC_DIRICHELET) return dir(ay(i, j, neg ? 0 : nz - 1), v);
    if (t == OCU_BC_NEUMANN) return neg ? ay(i, j, 0) - hz * (T)v : ay(i, j, nz - 1) + hz * (T)v;
    return mem(i, j, k);
  }
};

}  // namespace ocub
