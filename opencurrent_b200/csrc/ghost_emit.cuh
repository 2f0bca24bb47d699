// Ghost writes fused into the kernels that update interior cells.
#pragma once

#include "bc_device.cuh"

namespace ocub {

// Every ghost cell of the level1 fill is the x-, then y-, then z-rule applied to exactly one
// interior "source" cell (grid3dboundary.cu:237-347): a Dirichlet/Neumann ghost's source is the
// adjacent boundary cell, a periodic ghost's source is the cell on the opposite face, and
// edge/corner ghosts compose those per axis.  So the thread that writes the final value of an
// interior cell can also write every ghost that has that cell as its source, with the same
// arithmetic as the separate ghost-fill kernel -- the result is bit-identical to running the
// fill afterwards, and one launch per operation is saved.
//
// This is exact for colour sweeps too: a Dirichlet/Neumann ghost is read only by its own
// source cell, and a periodic ghost written during the red sweep is exactly the value the
// reference's between-colour refresh would produce (sol_mgpressure3ddev.cu:236-241).  It is
// not used when a face is BC_NONE (those ghosts keep stale values the composition reads).
template <typename T>
struct GhostEmit {
  T *p;
  long long xs, ys;
  int nx, ny, nz;
  BCDev bc;
  T hx, hy, hz;

  __device__ __forceinline__ int targets(int c, int n, int fneg, int fpos, int *idx, int *face) const {
    int m = 0;
    const int tn = bc.type[fneg], tp = bc.type[fpos];
    if ((tn == OCU_BC_DIRICHELET || tn == OCU_BC_NEUMANN) && c == 0) { idx[m] = -1; face[m] = fneg; m++; }
    else if (tn == OCU_BC_PERIODIC && c == n - 1) { idx[m] = -1; face[m] = fneg; m++; }
    if ((tp == OCU_BC_DIRICHELET || tp == OCU_BC_NEUMANN) && c == n - 1) { idx[m] = n; face[m] = fpos; m++; }
    else if (tp == OCU_BC_PERIODIC && c == 0) { idx[m] = n; face[m] = fpos; m++; }
    return m;
  }

  // face ids: odd = negative side (FX_NEG = 1, FY_NEG = 3, FZ_NEG = 5)
  __device__ __forceinline__ T rule(int f, T src, T h) const {
    const int t = bc.type[f];
    const float v = bc.value[f];
    if (t == OCU_BC_PERIODIC) return src;
    if (t == OCU_BC_DIRICHELET) return -src + (T)(2 * v);
    return (f & 1) ? src - h * (T)v : src + h * (T)v;
  }

  __device__ __forceinline__ void emit(int i, int j, int k, T val) const {
    if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) return;
    int xi[3], xf[3], yi[3], yf[3], zi[3], zf[3];
    xi[0] = i; yi[0] = j; zi[0] = k;
    xf[0] = yf[0] = zf[0] = 0;
    const int mx = 1 + targets(i, nx, FX_NEG, FX_POS, xi + 1, xf + 1);
    const int my = 1 + targets(j, ny, FY_NEG, FY_POS, yi + 1, yf + 1);
    const int mz = 1 + targets(k, nz, FZ_NEG, FZ_POS, zi + 1, zf + 1);
    for (int a = 0; a < mx; a++) {
      const T vx = a ? rule(xf[a], val, hx) : val;
      for (int b = 0; b < my; b++) {
        const T vy = b ? rule(yf[b], vx, hy) : vx;
        for (int c = 0; c < mz; c++) {
          if (a == 0 && b == 0 && c == 0) continue;
          const T vz = c ? rule(zf[c], vy, hz) : vy;
          p[(long long)xi[a] * xs + (long long)yi[b] * ys + zi[c]] = vz;
        }
      }
    }
  }
};

inline bool bc_has_none(const ocu_bc_set &b) {
  return b.xpos.type == OCU_BC_NONE || b.xneg.type == OCU_BC_NONE || b.ypos.type == OCU_BC_NONE ||
         b.yneg.type == OCU_BC_NONE || b.zpos.type == OCU_BC_NONE || b.zneg.type == OCU_BC_NONE;
}

}  // namespace ocub
