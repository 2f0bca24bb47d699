// FP32 correction solver of the refinement mixed solve (OCU_MG_MIXED_IR) on a red/black split
// ("chequer") layout.  No counterpart in the reference: the reference's mixed solver is an FP32
// warm start followed by FP64 multigrid (sol_mgpressuremixed3ddevd.cpp:79-100); here the FP32
// cycles are this library's own inner solver of an FP64 iterative refinement, checked against an
// FP64 multigrid solution at the requested tolerance rather than bit for bit.
//
// Layout: every level keeps, per colour c (cell (i,j,k) has colour (i+j+k)&1), one array of
// rows (i,j); cell k of row (i,j) in colour c sits at m = k >> 1 (the row holds the cells
// k = 2m + ((i+j+c)&1)).  Rows are rz floats long (rz = ceil(nz/2) rounded up to 4), no ghost
// cells: homogeneous boundary values are applied where a neighbour is read.  A colour sweep then
// reads the other colour's array and its own u and b, and writes its own u -- 2N*4 bytes -- where
// the interleaved layout moves 3N*4 (the two colours share every 32-byte sector).
#pragma once

#include <array>
#include <vector>

#include "ocu_internal.h"

namespace ocub {

struct ChqLevel {
  int nx, ny, nz, rz;
  double h;
  float *u[2], *b[2];
};

class ChequerMG {
 public:
  ~ChequerMG();
  // Whether the hierarchy can run here: at least two levels, every face Neumann, Dirichlet,
  // periodic or none, an even size along each periodic axis on every level, and a coarsest
  // level small enough for one CTA's shared memory (200 KB).
  static bool suits(const std::vector<std::array<int, 3>> &dims, const ocu_bc_set &bc);
  // dims / h: the FP64 hierarchy's levels; fx, fy, fz, omega: its operator factors.
  ocu_status init(const std::vector<std::array<int, 3>> &dims, const std::vector<double> &h, double fx,
                  double fy, double fz, double omega, const ocu_bc_set &bc_homogeneous);
  // Enqueue the correction solve from u(0) = 0: the right-hand side restricted to the coarsest
  // levels, solved there, carried up level by level with ramp_iters red-black iterations each
  // (nested iteration), then `cycles` V-cycles at level 0 (nu1 pre-smoothing iterations on every
  // level, nu2 post-smoothing on levels > 0, the coarsest level relaxed coarse_iters times).
  // With x (the FP64 level-0 grid at its interior origin, layout *Lx): then x += e, the last
  // prolongation adding into x directly where it can (u(0) is then left without it).
  ocu_status enqueue_fmg(int nu1, int nu2, int cycles, int coarse_iters, int ramp_iters, cudaStream_t s,
                         double *x = nullptr, const ocu_layout *Lx = nullptr);
  // Enqueue: b(0) = (float) (b - A x) from the FP64 level-0 grids (ghosts filled), with the
  // per-row sum of squares and max |r| of the FP64 residual in rows2 / rowsinf.
  ocu_status enqueue_residual(const double *x, const double *b, const ocu_layout &L, double h, double fx,
                              double fy, double fz, double *rows2, double *rowsinf, cudaStream_t s);
  // Enqueue: x += (double) u(0) on the interior.
  ocu_status enqueue_add_correction(double *x, const ocu_layout &L, cudaStream_t s);
  int levels() const { return (int)lv.size(); }
  // Single level operations on the stream (for testing and kernel timing): red-black iterations
  // (reverse = black first), one colour sweep, residual + restriction into level l + 1 (and its
  // u cleared), prolongation of level l into level l - 1.
  ocu_status relax_level(int l, int iterations, bool reverse, cudaStream_t s) { return relax(l, iterations, reverse, s); }
  ocu_status sweep_level(int l, int color, cudaStream_t s);
  ocu_status restrict_level(int l, cudaStream_t s) { return restrict_to(l, s); }
  ocu_status prolong_level(int l, cudaStream_t s) { return prolong_from(l, s); }
  const ChqLevel &level(int l) const { return lv[l]; }

 private:
  std::vector<ChqLevel> lv;
  void *block = nullptr;
  double fx = 1, fy = 1, fz = 1, omega = 1;
  ocu_bc_set bc{};
  ocu_status relax(int l, int iterations, bool reverse, cudaStream_t s);
  // zero_u: level l's u is zero and is not read (only b is restricted)
  ocu_status restrict_to(int l, cudaStream_t s, bool zero_u = false);
  // mode: CHQ_P_ADD / ASSIGN / X64 / X64V (chq_device.cuh); x, Lx for the X64 modes
  ocu_status prolong_from(int l, cudaStream_t s, int mode = 0, double *x = nullptr, const ocu_layout *Lx = nullptr);
  // levels tail_s..L-1 in one single-CTA launch: FMG (fmg) or one V-cycle from tail_s
  ocu_status tail(bool fmg, int nu1, int nu2, int citers, cudaStream_t s);
  int tail_s = 0;
};

}  // namespace ocub
