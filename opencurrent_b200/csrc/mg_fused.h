// Shared device-side pieces of the multigrid kernels (coefficients, coarsest-level block
// relaxation, single-CTA tail parameters) and the fused-kernel launchers.
#pragma once

#include "bc_device.cuh"
#include "ocu_internal.h"

namespace ocub {

// Colour-sweep coefficients rounded to T the way the reference launcher rounds them
// (sol_mgpressure3ddevf.cu:390-393 float, sol_mgpressure3ddevd.cu:1262-1268 double).
template <typename T>
struct RelaxCoefD {
  T omega, hsq, fx, fy, fz, ld;  // hsq = (T)(h*h) for float, (-h)*h for double
  T xp, xn, yp, yn, zp, zn;
};

template <typename T>
inline RelaxCoefD<T> make_relax_coef_d(const RelaxParams &p) {
  RelaxCoefD<T> c;
  c.omega = (T)p.omega;
  c.hsq = sizeof(T) == 4 ? (T)(p.h * p.h) : (T)(-p.h * p.h);
  c.fx = (T)p.fx; c.fy = (T)p.fy; c.fz = (T)p.fz;
  c.ld = (T)(2 * p.fx + 2 * p.fy + 2 * p.fz);
  c.xp = (T)bc_diag_mod(p.bc.xpos, p.fx); c.xn = (T)bc_diag_mod(p.bc.xneg, p.fx);
  c.yp = (T)bc_diag_mod(p.bc.ypos, p.fy); c.yn = (T)bc_diag_mod(p.bc.yneg, p.fy);
  c.zp = (T)bc_diag_mod(p.bc.zpos, p.fz); c.zn = (T)bc_diag_mod(p.bc.zneg, p.fz);
  return c;
}

// do_cpu_solve coefficients (sol_mgpressure3ddev.cu:82-125)
template <typename T>
struct CoarseCoef {
  double fx, fy, fz;
  T omega, ld, h;
  T xp, xn, yp, yn, zp, zn;
};

template <typename T>
inline CoarseCoef<T> make_coarse_coef(const RelaxParams &p) {
  CoarseCoef<T> c;
  c.fx = p.fx; c.fy = p.fy; c.fz = p.fz;
  c.omega = (T)p.omega;
  c.ld = (T)(2 * p.fx + 2 * p.fy + 2 * p.fz);
  c.h = (T)p.h;
  c.xp = (T)bc_diag_mod(p.bc.xpos, p.fx); c.xn = (T)bc_diag_mod(p.bc.xneg, p.fx);
  c.yp = (T)bc_diag_mod(p.bc.ypos, p.fy); c.yn = (T)bc_diag_mod(p.bc.yneg, p.fy);
  c.zp = (T)bc_diag_mod(p.bc.zpos, p.fz); c.zn = (T)bc_diag_mod(p.bc.zneg, p.fz);
  return c;
}

template <typename T>
__device__ __forceinline__ T host_face(const BCDev &bc, int f, T src, T h, bool neg) {
  const int t = bc.ty(f);
  if (t == OCU_BC_DIRICHELET) return -src + (T)2 * (T)bc.val(f);
  if (t == OCU_BC_NEUMANN) return neg ? src - h * (T)bc.val(f) : src + h * (T)bc.val(f);
  return src;
}

// Coarsest-level relaxation as the reference runs it on the host: do_cpu_solve per colour
// (the _fz*(...) products in double, accumulated into a T residual), the host faces-only ghost
// fill in T after every colour (grid3dboundary.cu:1018-1111), and the device level1 fill at the
// end (sol_mgpressure3ddev.cu:134-188).  Executed by one thread block, phases separated by
// __syncthreads; the caller has already adjusted `iterations` for RO_SYMMETRIC.
template <typename T>
__device__ void coarse_relax_block(T *u, const T *b, long long xs, long long ys, int nx, int ny, int nz,
                                   int iterations, int order, const CoarseCoef<T> &c, const BCDev &bc, T hx,
                                   T hy, T hz) {
  const int nt = blockDim.x;
  const int ncell = nx * ny * nz;
  auto at = [&](int i, int j, int k) -> T & { return u[(long long)i * xs + (long long)j * ys + k]; };
  const int nzf = nx * ny, nyf = nx * nz, nxf = ny * nz, nghost = 2 * (nzf + nyf + nxf);
  if (ncell <= nt && nghost <= nt) {
    // every thread owns at most one cell and one face ghost: their indices, diagonal and ghost
    // rule are worked out once, and each of the 4 phases of an iteration is a short chain
    const int q = threadIdx.x;
    const bool own = q < ncell;
    int i = 0, j = 0, k = 0;
    long long id = 0;
    T dg = c.ld;
    if (own) {
      i = q / (ny * nz), j = (q / nz) % ny, k = q % nz;
      id = (long long)i * xs + (long long)j * ys + k;
      const T x_mod = (i == 0) ? c.xn : (i == nx - 1) ? c.xp : (T)0;
      const T y_mod = (j == 0) ? c.yn : (j == ny - 1) ? c.yp : (T)0;
      const T z_mod = (k == 0) ? c.zn : (k == nz - 1) ? c.zp : (T)0;
      dg = c.ld + x_mod + y_mod + z_mod;
    }
    // ghost item: dst <- src (periodic copy) or host_face(src) (Dirichlet / Neumann)
    int gkind = 0, gf = 0;  // 0 none, 1 copy, 2 rule
    long long gdst = 0, gsrc = 0;
    T gh = 0;
    bool gneg = false;
    if (q < nghost) {
      int r = q, gi, gj, gk, si, sj, sk;
      if (r < 2 * nzf) {
        const int side = r / nzf;
        gi = si = (r % nzf) / ny, gj = sj = (r % nzf) % ny;
        gf = side ? FZ_POS : FZ_NEG, gh = hz, gneg = !side;
        gk = side ? nz : -1;
        sk = bc.ty(gf) == OCU_BC_PERIODIC ? (side ? 0 : nz - 1) : (side ? nz - 1 : 0);
      } else if ((r -= 2 * nzf) < 2 * nyf) {
        const int side = r / nyf;
        gi = si = (r % nyf) / nz, gk = sk = (r % nyf) % nz;
        gf = side ? FY_POS : FY_NEG, gh = hy, gneg = !side;
        gj = side ? ny : -1;
        sj = bc.ty(gf) == OCU_BC_PERIODIC ? (side ? 0 : ny - 1) : (side ? ny - 1 : 0);
      } else {
        r -= 2 * nyf;
        const int side = r / nxf;
        gj = sj = (r % nxf) / nz, gk = sk = (r % nxf) % nz;
        gf = side ? FX_POS : FX_NEG, gh = hx, gneg = !side;
        gi = side ? nx : -1;
        si = bc.ty(gf) == OCU_BC_PERIODIC ? (side ? 0 : nx - 1) : (side ? nx - 1 : 0);
      }
      const int t = bc.ty(gf);
      gkind = t == OCU_BC_PERIODIC ? 1 : (t == OCU_BC_DIRICHELET || t == OCU_BC_NEUMANN) ? 2 : 0;
      gdst = (long long)gi * xs + (long long)gj * ys + gk;
      gsrc = (long long)si * xs + (long long)sj * ys + sk;
    }
    for (int it = 0; it < iterations; it++) {
      for (int rb = 0; rb < 2; rb++) {
        int color = rb;
        if (order == 1 || (order == 2 && it >= iterations / 2)) color = !rb;
        if (own && ((i + j + color) & 1) == (k & 1)) {
          T residual = (-c.h * c.h * b[id] - c.ld * u[id]);
          residual = (T)((double)residual + c.fz * (double)(u[id - 1] + u[id + 1]));
          residual = (T)((double)residual + c.fy * (double)(u[id + ys] + u[id - ys]));
          residual = (T)((double)residual + c.fx * (double)(u[id + xs] + u[id - xs]));
          u[id] = u[id] + c.omega * residual / dg;
        }
        __syncthreads();
        if (gkind == 1) u[gdst] = u[gsrc];
        else if (gkind == 2) u[gdst] = host_face<T>(bc, gf, u[gsrc], gh, gneg);
        __syncthreads();
      }
    }
    level1_fill_block<T>(u, xs, ys, nx, ny, nz, bc, hx, hy, hz);
    __syncthreads();
    return;
  }
  for (int it = 0; it < iterations; it++) {
    for (int rb = 0; rb < 2; rb++) {
      int color = rb;
      if (order == 1 || (order == 2 && it >= iterations / 2)) color = !rb;
      for (int q = threadIdx.x; q < ncell; q += nt) {
        const int i = q / (ny * nz), j = (q / nz) % ny, k = q % nz;
        if (((i + j + color) & 1) != (k & 1)) continue;
        const long long id = (long long)i * xs + (long long)j * ys + k;
        const T x_mod = (i == 0) ? c.xn : (i == nx - 1) ? c.xp : (T)0;
        const T y_mod = (j == 0) ? c.yn : (j == ny - 1) ? c.yp : (T)0;
        const T z_mod = (k == 0) ? c.zn : (k == nz - 1) ? c.zp : (T)0;
        T residual = (-c.h * c.h * b[id] - c.ld * u[id]);
        residual = (T)((double)residual + c.fz * (double)(u[id - 1] + u[id + 1]));
        residual = (T)((double)residual + c.fy * (double)(u[id + ys] + u[id - ys]));
        residual = (T)((double)residual + c.fx * (double)(u[id + xs] + u[id - xs]));
        u[id] = u[id] + c.omega * residual / (c.ld + x_mod + y_mod + z_mod);
      }
      __syncthreads();
      for (int q = threadIdx.x; q < nghost; q += nt) {
        int r = q;
        if (r < 2 * nzf) {
          const int side = r / nzf, i = (r % nzf) / ny, j = (r % nzf) % ny;
          const int f = side ? FZ_POS : FZ_NEG, t = bc.ty(f);
          if (t == OCU_BC_PERIODIC) at(i, j, side ? nz : -1) = at(i, j, side ? 0 : nz - 1);
          else if (t == OCU_BC_DIRICHELET || t == OCU_BC_NEUMANN)
            at(i, j, side ? nz : -1) = host_face<T>(bc, f, at(i, j, side ? nz - 1 : 0), hz, !side);
          continue;
        }
        r -= 2 * nzf;
        if (r < 2 * nyf) {
          const int side = r / nyf, i = (r % nyf) / nz, k = (r % nyf) % nz;
          const int f = side ? FY_POS : FY_NEG, t = bc.ty(f);
          if (t == OCU_BC_PERIODIC) at(i, side ? ny : -1, k) = at(i, side ? 0 : ny - 1, k);
          else if (t == OCU_BC_DIRICHELET || t == OCU_BC_NEUMANN)
            at(i, side ? ny : -1, k) = host_face<T>(bc, f, at(i, side ? ny - 1 : 0, k), hy, !side);
          continue;
        }
        r -= 2 * nyf;
        {
          const int side = r / nxf, j = (r % nxf) / nz, k = (r % nxf) % nz;
          const int f = side ? FX_POS : FX_NEG, t = bc.ty(f);
          if (t == OCU_BC_PERIODIC) at(side ? nx : -1, j, k) = at(side ? 0 : nx - 1, j, k);
          else if (t == OCU_BC_DIRICHELET || t == OCU_BC_NEUMANN)
            at(side ? nx : -1, j, k) = host_face<T>(bc, f, at(side ? nx - 1 : 0, j, k), hx, !side);
        }
      }
      __syncthreads();
    }
  }
  level1_fill_block<T>(u, xs, ys, nx, ny, nz, bc, hx, hy, hz);
  __syncthreads();
}

template <typename T>
struct ResCoefT {
  T fxh, fyh, fzh, dg;
};

// One level of the single-CTA tail.
template <typename T>
struct TailLevel {
  T *u;
  T *b;
  long long xs, ys;
  int nx, ny, nz;
  int emit_ok;  // ghosts may be written by the sweeping threads (no BC_NONE, even periodic axes)
  int periodic; // any periodic face (ghost refresh between colours when emit_ok == 0)
  BCDev bc;
  T hx, hy, hz;
  RelaxCoefD<T> rc;
  ResCoefT<T> res;
};

constexpr int kMaxTailLevels = 8;

template <typename T>
struct TailParams {
  TailLevel<T> lv[kMaxTailLevels];
  int nlev;          // levels in the tail; lv[nlev-1] is the coarsest
  int first_level;   // absolute level number of lv[0]
  int nu1, nu2;
  int post_order;    // relax order of the up-leg (RO_BLACK_RED when symmetric)
  int coarse_iters;  // already adjusted for RO_SYMMETRIC when host_coarse
  int coarse_order;
  int host_coarse;   // 1: coarsest relaxed with the host routine's arithmetic
  CoarseCoef<T> cc;
};

// Member selection of the ensemble (batched) launches: member m of a level lives at
// base + m * stride; a launch processes the members whose state equals `want`.  state ==
// nullptr: a single grid (member 0 only).
struct BatchSel {
  const int *state;
  int want;
};
struct TailBatch {
  BatchSel sel;
  long long ms[kMaxTailLevels];  // member stride of each tail level (elements)
};

template <typename T>
ocu_status launch_relax_color_emit(T *u, const T *b, const ocu_layout &L, const T *diag, int color,
                                   const RelaxParams &p, double hx, double hy, double hz, cudaStream_t s);
template <typename T>
ocu_status launch_prolong_emit(const T *uc, const ocu_layout &Lc, T *uf, const ocu_layout &Lf,
                               const ocu_bc_set &bc_fine, double hx, double hy, double hz, cudaStream_t s);
template <typename T>
ocu_status launch_residual_rows(const T *u, const T *b, T *r, float *r32, const ocu_layout &L, double h, double fx,
                                double fy, double fz, T *rows2, T *rowsinf, cudaStream_t s);
template <typename T>
ocu_status launch_residual_restrict(const T *u, const T *b, const ocu_layout &Lf, T *bc_, const ocu_layout &Lc,
                                    double h, double fx, double fy, double fz, T *rows2, T *rowsinf, cudaStream_t s,
                                    T *zero_u = nullptr, long long zero_n = 0);
template <typename T>
ocu_status launch_fold_rows(const T *rows, long long nrows, bool is_max, void *scratch, double *result,
                            cudaStream_t s);
template <typename T>
ocu_status launch_coarse_tail(const TailParams<T> &P, cudaStream_t s);
// The same schedule for `members` grids at once, one CTA per member.
// The tail over the CTAs of one cluster (2..8 CTAs; every tail level with fused ghost writes).
template <typename T>
ocu_status launch_coarse_tail_batch(const TailParams<T> &P, const TailBatch &tb, int members, cudaStream_t s);

// Ensemble forms of the level kernels over `members` congruent grids (member m at base + m*ms;
// ms, fms, cms are member strides in elements).  See kernels_mg_fused.cu.
template <typename T>
ocu_status launch_relax_color_emit_b(T *u, const T *b, const ocu_layout &L, const T *diag, int color,
                                     const RelaxParams &p, double hx, double hy, double hz, const BatchSel &sel,
                                     long long ms, int members, const int block[3], cudaStream_t s);
template <typename T>
ocu_status launch_prolong_emit_b(const T *uc, const ocu_layout &Lc, T *uf, const ocu_layout &Lf,
                                 const ocu_bc_set &bc_fine, double hx, double hy, double hz, const BatchSel &sel,
                                 long long cms, long long fms, int members, cudaStream_t s);
template <typename T>
ocu_status launch_residual_restrict_b(const T *u, const T *b, const ocu_layout &Lf, T *bc_, const ocu_layout &Lc,
                                      double h, double fx, double fy, double fz, T *rows2, const BatchSel &sel,
                                      long long fms, long long cms, int members, cudaStream_t s);
template <typename T>
ocu_status launch_residual_rows_b(const T *u, const T *b, const ocu_layout &L, double h, double fx, double fy,
                                  double fz, T *rows2, const BatchSel &sel, long long ms, int members,
                                  cudaStream_t s);
template <typename T>
ocu_status launch_fold_rows_b(const T *rows, long long nrows, T *partial, long long pstride, double *sums,
                              const BatchSel &sel, int members, cudaStream_t s);
template <typename T>
ocu_status launch_bc_fill_b(T *u, const ocu_layout &L, const ocu_bc_set &bc, double hx, double hy, double hz,
                            const BatchSel &sel, long long ms, int members, int *state, bool retire,
                            cudaStream_t s);
template <typename T>
ocu_status launch_converge_b(const double *sums, long long ncell, const double *tol, int *state, int *vcycles,
                             double *last_l2, int *active, int members, bool initial, cudaStream_t s);

// Opaque copy of a CUtensorMap (128 bytes, 64-byte aligned) so host headers need no cuda.h.
struct alignas(64) SweepTmap {
  unsigned char bytes[128];
};
// Two-colour sweep (kernels_relax_tma.cu): supported layouts/BCs, the tensor map of one grid
// buffer, and the launch u_in (through its map) -> u_out.  err: device word set to 1 when a
// bounded wait inside the kernel gives up; wait_limit: polls before a wait gives up (0 = the
// default, about a second; negative = the timeout test, see ocu_mg_params.wait_limit).
bool sweep2_supported(const ocu_layout &L, const ocu_bc_set &bc);
template <typename T>
ocu_status make_sweep_tmap(const void *buf, const ocu_layout &L, SweepTmap *out);
template <typename T>
ocu_status launch_relax_sweep2(const SweepTmap &tm_u_in, const SweepTmap &tm_b, T *u_out, const ocu_layout &L,
                               const T *diag, int first_color, const RelaxParams &p, double hx, double hy, double hz,
                               int *err, cudaStream_t s, int wait_limit = 0);

}  // namespace ocub
