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

  // Does the negative (resp. positive) face of an axis take coordinate c as a ghost source?
  __device__ __forceinline__ bool src_neg(int t, int c, int n) const {
    return ((t == OCU_BC_DIRICHELET || t == OCU_BC_NEUMANN) && c == 0) || (t == OCU_BC_PERIODIC && c == n - 1);
  }
  __device__ __forceinline__ bool src_pos(int t, int c, int n) const {
    return ((t == OCU_BC_DIRICHELET || t == OCU_BC_NEUMANN) && c == n - 1) || (t == OCU_BC_PERIODIC && c == 0);
  }

  // face ids: odd = negative side (FX_NEG = 1, FY_NEG = 3, FZ_NEG = 5)
  template <int F>
  __device__ __forceinline__ T rule(T src, T h) const {
    const int t = bc.type[F];
    const float v = bc.value[F];
    if (t == OCU_BC_PERIODIC) return src;
    if (t == OCU_BC_DIRICHELET) return -src + (T)(2 * v);
    return (F & 1) ? src - h * (T)v : src + h * (T)v;
  }

  // Writes every ghost whose source is (i,j,k): per axis the candidates are the cell itself,
  // the negative-face ghost and the positive-face ghost, composed x -> y -> z.  The loops are
  // fully unrolled so every face index is a constant (per-thread local arrays, or a face index
  // known only at run time, would put the struct in local memory for every thread).
  __device__ __forceinline__ void emit(int i, int j, int k, T val) const {
    if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) return;
    const bool x1 = src_neg(bc.type[FX_NEG], i, nx), x2 = src_pos(bc.type[FX_POS], i, nx);
    const bool y1 = src_neg(bc.type[FY_NEG], j, ny), y2 = src_pos(bc.type[FY_POS], j, ny);
    const bool z1 = src_neg(bc.type[FZ_NEG], k, nz), z2 = src_pos(bc.type[FZ_POS], k, nz);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if ((a == 1 && !x1) || (a == 2 && !x2)) continue;
      const T vx = a == 0 ? val : a == 1 ? rule<FX_NEG>(val, hx) : rule<FX_POS>(val, hx);
      const long long ox = (long long)(a == 0 ? i : a == 1 ? -1 : nx) * xs;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        if ((b == 1 && !y1) || (b == 2 && !y2)) continue;
        const T vy = b == 0 ? vx : b == 1 ? rule<FY_NEG>(vx, hy) : rule<FY_POS>(vx, hy);
        const long long oy = ox + (long long)(b == 0 ? j : b == 1 ? -1 : ny) * ys;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          if (a == 0 && b == 0 && c == 0) continue;
          if ((c == 1 && !z1) || (c == 2 && !z2)) continue;
          const T vz = c == 0 ? vy : c == 1 ? rule<FZ_NEG>(vy, hz) : rule<FZ_POS>(vy, hz);
          p[oy + (c == 0 ? k : c == 1 ? -1 : nz)] = vz;
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
