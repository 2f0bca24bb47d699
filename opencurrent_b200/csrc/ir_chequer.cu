// FP32 correction solver of the refinement mixed solve on the red/black split layout (see
// ir_chequer.h).  This is the library's own inner solver, not a reference routine: its operator,
// smoother and transfer operators are the reference multigrid's (7-point operator with the
// reference's boundary diagonal modifications, Yavneh-omega red-black SOR, 8-cell restriction,
// trilinear prolongation; sol_mgpressure3ddevf.cu:38-252), evaluated with fused multiply-adds
// and a precomputed omega/diagonal, and checked against an FP64 multigrid solution instead of
// bit for bit.
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "chq_device.cuh"
#include "mg_fused.h"

namespace ocub {

using namespace chq;

namespace {

__global__ void __launch_bounds__(CHQ_RELAX_THREADS) k_chq_relax(ChqG g, ChqK k, ChqBC bc, int color) {
  pdl_entry();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)g.nx * g.ny * (g.rz >> 2)) return;
  chq_relax_item<true>(g, k, bc, color, (int)t);
}

template <bool ZU>
__global__ void __launch_bounds__(256, CHQ_RESTRICT_MINB) k_chq_restrict(ChqG f, ChqG c, ChqK k, ChqBC bc, FDiv fcm) {
  pdl_entry();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)c.nx * c.ny * fcm.d) return;
  chq_restrict_item<true, ZU>(f, c, k, bc, fcm, (int)t);
}

template <int MODE>
__global__ void __launch_bounds__(256, CHQ_PROLONG_MINB) k_chq_prolong(ChqG c, ChqG f, ChqBC bc, FDiv fcm, ChqX X) {
  pdl_entry();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)c.nx * c.ny * fcm.d) return;
  chq_prolong_item<true, MODE>(c, f, bc, fcm, (int)t, X);
}

__global__ void __launch_bounds__(1024) k_chq_tail(ChqTail T) {
  pdl_entry();
  extern __shared__ float sm[];
  __shared__ SLv lv[kChqMaxTail];
  if (threadIdx.x == 0) {
#pragma unroll
    for (int l = 0; l < kChqMaxTail; l++)
      if (l < T.nlev) lv[l] = T.lv[l];
  }
  __syncthreads();
  chq_tail_run(T, lv, sm);
}

// FP64 residual of the refinement step, written as float into the level-0 colour arrays, with
// per-row sum of squares and max |r| (one warp per row (i, j)).
struct OuterCoef {
  double fxh, fyh, fzh, dg;
};

template <bool VEC>
__global__ void __launch_bounds__(256) k_chq_outer_residual(const double *__restrict__ x, const double *__restrict__ b,
                                                            long long xs, long long ys, int nx, int ny, int nz,
                                                            OuterCoef c, float *__restrict__ B0,
                                                            float *__restrict__ B1, int rz,
                                                            double *__restrict__ rows2,
                                                            double *__restrict__ rowsinf) {
  pdl_entry();
  const int lane = threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (j >= ny) return;  // whole warp
  const long long row = (long long)i * xs + (long long)j * ys;
  const long long crow = ((long long)i * ny + j) * rz;
  const bool s = (i + j) & 1;
  float *__restrict__ Bs = s ? B1 : B0;
  float *__restrict__ Bo = s ? B0 : B1;
  double acc2 = 0, accinf = 0;
  for (int m = lane; 2 * m < nz; m += 32) {
    if (VEC) {  // nz even, rows on 16-byte boundaries: the pair and its neighbours as double2
      const long long id = row + 2 * m;
      const double2 X = *reinterpret_cast<const double2 *>(x + id), B = *reinterpret_cast<const double2 *>(b + id);
      const double2 YM = *reinterpret_cast<const double2 *>(x + id - ys), YP = *reinterpret_cast<const double2 *>(x + id + ys);
      const double2 XM = *reinterpret_cast<const double2 *>(x + id - xs), XP = *reinterpret_cast<const double2 *>(x + id + xs);
      const double zl = x[id - 1], zr = x[id + 2];
      const double r0 = B.x - (c.fzh * (zl + X.y) + c.fyh * (YM.x + YP.x) + c.fxh * (XM.x + XP.x) - c.dg * X.x);
      const double r1 = B.y - (c.fzh * (X.x + zr) + c.fyh * (YM.y + YP.y) + c.fxh * (XM.y + XP.y) - c.dg * X.y);
      Bs[crow + m] = (float)r0;
      Bo[crow + m] = (float)r1;
      acc2 += r0 * r0 + r1 * r1;
      accinf = fmax(accinf, fmax(fabs(r0), fabs(r1)));
      continue;
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int k = 2 * m + h;
      if (k < nz) {
        const long long id = row + k;
        const double r = b[id] - (c.fzh * (x[id - 1] + x[id + 1]) + c.fyh * (x[id - ys] + x[id + ys]) +
                                  c.fxh * (x[id - xs] + x[id + xs]) - c.dg * x[id]);
        (h ? Bo : Bs)[crow + m] = (float)r;
        acc2 += r * r;
        accinf = fmax(accinf, fabs(r));
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc2 += __shfl_down_sync(0xffffffffu, acc2, o);
    accinf = fmax(accinf, __shfl_down_sync(0xffffffffu, accinf, o));
  }
  if (lane == 0) {
    rows2[(long long)i * ny + j] = acc2;
    rowsinf[(long long)i * ny + j] = accinf;
  }
}

// x += (double) e on the interior, e on the level-0 colour arrays.
template <bool VEC>
__global__ void __launch_bounds__(256) k_chq_add_correction(double *__restrict__ x, long long xs, long long ys,
                                                            int nx, int ny, int nz, const float *__restrict__ E0,
                                                            const float *__restrict__ E1, int rz) {
  pdl_entry();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (j >= ny || 2 * m >= nz) return;
  const long long id = (long long)i * xs + (long long)j * ys + 2 * m;
  const long long cid = ((long long)i * ny + j) * rz + m;
  const bool s = (i + j) & 1;
  const float e0 = (s ? E1 : E0)[cid], e1 = (s ? E0 : E1)[cid];
  if (VEC) {
    double2 X = *reinterpret_cast<double2 *>(x + id);
    X.x = X.x + (double)e0;
    X.y = X.y + (double)e1;
    *reinterpret_cast<double2 *>(x + id) = X;
    return;
  }
  x[id] = x[id] + (double)e0;
  if (2 * m + 1 < nz) x[id + 1] = x[id + 1] + (double)e1;
}

}  // namespace

// the FP64 grid's pairs (k, k+1), k even, are 16-byte aligned double2
static bool vec_ok(const ocu_layout &L) {
  return L.nz % 2 == 0 && L.shift % 2 == 0 && L.xstride % 2 == 0 && L.ystride % 2 == 0;
}

bool ChequerMG::suits(const std::vector<std::array<int, 3>> &dims, const ocu_bc_set &bc) {
  if (dims.size() < 2) return false;
  const ocu_bc *f[6] = {&bc.xpos, &bc.xneg, &bc.ypos, &bc.yneg, &bc.zpos, &bc.zneg};
  for (int q = 0; q < 6; q++) {
    const int t = f[q]->type;
    if (t != OCU_BC_NEUMANN && t != OCU_BC_DIRICHELET && t != OCU_BC_PERIODIC && t != OCU_BC_NONE) return false;
  }
  // a periodic axis must be periodic on both faces and even on every level (the colouring
  // then continues across the wrap)
  const bool per[3] = {bc.xpos.type == OCU_BC_PERIODIC, bc.ypos.type == OCU_BC_PERIODIC,
                       bc.zpos.type == OCU_BC_PERIODIC};
  const bool per_neg[3] = {bc.xneg.type == OCU_BC_PERIODIC, bc.yneg.type == OCU_BC_PERIODIC,
                           bc.zneg.type == OCU_BC_PERIODIC};
  for (int a = 0; a < 3; a++) {
    if (per[a] != per_neg[a]) return false;
    if (per[a])
      for (const auto &d : dims)
        if (d[a] % 2) return false;
  }
  for (const auto &d : dims)
    if ((long long)d[0] * d[1] * round4((d[2] + 1) / 2) / 4 >= (1LL << 31) / 8) return false;
  return level_smem(dims.back()) <= kTailSmemCap;
}

ChequerMG::~ChequerMG() {
  if (block) cudaFree(block);
}

ocu_status ChequerMG::init(const std::vector<std::array<int, 3>> &dims, const std::vector<double> &h, double fx_,
                           double fy_, double fz_, double omega_, const ocu_bc_set &bc_h) {
  fx = fx_; fy = fy_; fz = fz_; omega = omega_; bc = bc_h;
  lv.clear();
  size_t total = 0;
  for (size_t l = 0; l < dims.size(); l++) {
    ChqLevel L{};
    L.nx = dims[l][0]; L.ny = dims[l][1]; L.nz = dims[l][2];
    L.rz = round4((L.nz + 1) / 2);
    L.h = h[l];
    lv.push_back(L);
    total += 4 * (size_t)L.nx * L.ny * L.rz;
  }
  tail_s = tail_first(dims, tail_cells_setting());
  size_t tail_bytes = 0;
  for (size_t l = tail_s; l < dims.size(); l++) tail_bytes += level_smem(dims[l]);
  OCU_TRY(check_cuda(cudaFuncSetAttribute(k_chq_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTailSmemCap),
                     "cudaFuncSetAttribute (tail kernel)"));
  (void)tail_bytes;
  OCU_TRY(check_cuda(cudaMalloc(&block, total * sizeof(float)), "cudaMalloc (FP32 refinement levels)"));
  OCU_TRY(check_cuda(cudaMemset(block, 0, total * sizeof(float)), "cudaMemset"));
  float *p = (float *)block;
  for (auto &L : lv) {
    const size_t n = (size_t)L.nx * L.ny * L.rz;
    L.u[0] = p; L.u[1] = p + n; L.b[0] = p + 2 * n; L.b[1] = p + 3 * n;
    p += 4 * n;
  }
  return OCU_OK;
}

ocu_status ChequerMG::relax(int l, int iterations, bool reverse, cudaStream_t s) {
  const ChqLevel &L = lv[l];
  const ChqG g = make_g(L);
  const ChqK k = make_k(L.h, fx, fy, fz, omega);
  const ChqBC b = make_bc(bc, fx, fy, fz);
  const long long threads = (long long)L.nx * L.ny * (L.rz / 4);
  const int blocks = (int)((threads + CHQ_RELAX_THREADS - 1) / CHQ_RELAX_THREADS);
  for (int it = 0; it < iterations; it++)
    for (int h = 0; h < 2; h++) {
      launch_pdl(k_chq_relax, dim3(blocks), dim3(CHQ_RELAX_THREADS), 0, s, g, k, b, reverse ? 1 - h : h);
      OCU_TRY(check_launch("k_chq_relax"));
    }
  return OCU_OK;
}

ocu_status ChequerMG::sweep_level(int l, int color, cudaStream_t s) {
  const ChqLevel &L = lv[l];
  const long long threads = (long long)L.nx * L.ny * (L.rz / 4);
  launch_pdl(k_chq_relax, dim3((unsigned)((threads + CHQ_RELAX_THREADS - 1) / CHQ_RELAX_THREADS)),
             dim3(CHQ_RELAX_THREADS), 0, s, make_g(L),
             make_k(L.h, fx, fy, fz, omega), make_bc(bc, fx, fy, fz), color & 1);
  return check_launch("k_chq_relax");
}

ocu_status ChequerMG::restrict_to(int l, cudaStream_t s, bool zero_u) {
  const ChqLevel &F = lv[l], &Cl = lv[l + 1];
  const int cm = (Cl.nz + 1) / 2;  // coarse pairs per row
  const long long n = (long long)Cl.nx * Cl.ny * cm;
  const dim3 grid((unsigned)((n + 255) / 256));
  if (zero_u)
    launch_pdl(k_chq_restrict<true>, grid, dim3(256), 0, s, make_g(F), make_g(Cl), make_k(F.h, fx, fy, fz, omega),
               make_bc(bc, fx, fy, fz), make_fdiv(cm));
  else
    launch_pdl(k_chq_restrict<false>, grid, dim3(256), 0, s, make_g(F), make_g(Cl), make_k(F.h, fx, fy, fz, omega),
               make_bc(bc, fx, fy, fz), make_fdiv(cm));
  return check_launch("k_chq_restrict");
}

ocu_status ChequerMG::prolong_from(int l, cudaStream_t s, int mode, double *x, const ocu_layout *Lx) {
  const ChqLevel &Cl = lv[l], &F = lv[l - 1];
  const int cm = (Cl.nz + 1) / 2;
  const long long n = (long long)Cl.nx * Cl.ny * cm;
  const dim3 grid((unsigned)((n + 255) / 256));
  ChqX X{x, Lx ? (long long)Lx->xstride : 0, Lx ? (long long)Lx->ystride : 0};
  const ChqG cg = make_g(Cl), fg = make_g(F);
  const ChqBC b = make_bc(bc, fx, fy, fz);
  const FDiv d = make_fdiv(cm);
  switch (mode) {
    case CHQ_P_ASSIGN: launch_pdl(k_chq_prolong<CHQ_P_ASSIGN>, grid, dim3(256), 0, s, cg, fg, b, d, X); break;
    case CHQ_P_X64: launch_pdl(k_chq_prolong<CHQ_P_X64>, grid, dim3(256), 0, s, cg, fg, b, d, X); break;
    case CHQ_P_X64V: launch_pdl(k_chq_prolong<CHQ_P_X64V>, grid, dim3(256), 0, s, cg, fg, b, d, X); break;
    default: launch_pdl(k_chq_prolong<CHQ_P_ADD>, grid, dim3(256), 0, s, cg, fg, b, d, X); break;
  }
  return check_launch("k_chq_prolong");
}

ocu_status ChequerMG::tail(bool fmg, int nu1, int nu2, int citers, cudaStream_t s) {
  ChqTail T{};
  const int L = levels();
  T.nlev = L - tail_s;
  T.nu1 = nu1; T.nu2 = nu2; T.citers = citers;
  T.level0 = tail_s == 0;
  T.fmg = fmg ? 1 : 0;
  T.bc = make_bc(bc, fx, fy, fz);
  int off = 0, largest = 0;
  for (int l = tail_s; l < L; l++) {
    const ChqLevel &C = lv[l];
    SLv &d = T.lv[l - tail_s];
    d.nx = C.nx; d.ny = C.ny; d.nz = C.nz; d.rz = C.rz;
    d.off = off;
    d.mlog = log2_exact((C.nz + 1) / 2);
    d.ylog = log2_exact(C.ny);
    d.nzlog = log2_exact(C.nz);
    d.k = make_k(C.h, fx, fy, fz, omega);
    d.gu0 = C.u[0]; d.gu1 = C.u[1]; d.gb0 = C.b[0]; d.gb1 = C.b[1];
    off += 4 * C.nx * C.ny * C.rz;
    if (l < L - 1 && 2 * C.nx * C.ny * C.rz > largest) largest = 2 * C.nx * C.ny * C.rz;
  }
  T.scratch = off;
  off += largest;
  // threads: enough for the largest phase of the top level, in whole warps, at most 1024
  const ChqLevel &top = lv[tail_s];
  const long long work = (long long)top.nx * top.ny * top.nz;
  const int threads = (int)std::min<long long>(1024, std::max<long long>(64, ((work + 31) / 32) * 32));
  launch_pdl(k_chq_tail, dim3(1), dim3(threads), (size_t)off * sizeof(float), s, T);
  return check_launch("k_chq_tail");
}

// Nested iteration + V-cycles: the right-hand side restricted down to the tail, the tail
// levels solved in one launch, then on the way up each level gets the prolonged coarse solution
// and ramp_iters red-black iterations (no V-cycle: measured at 256^3, a refinement solve takes
// 3.87 ms this way against 4.61 ms with one V-cycle per ramp level, at the same residual after
// the same two refinement steps), and level 0 gets `cycles` V-cycles.
// The correction starts from zero, so the first descent restricts b alone (the residual of a
// zero u is b) and each level's first prolongation assigns instead of adding: level 0 is never
// cleared or read before it is written.  With x given, the last prolongation into level 0 adds
// e + p/64 to x (in double) instead of storing it -- level 0 then does not hold the final
// correction -- otherwise x += e follows as its own pass.
ocu_status ChequerMG::enqueue_fmg(int nu1, int nu2, int cycles, int coarse_iters, int ramp_iters, cudaStream_t s,
                                  double *x, const ocu_layout *Lx) {
  const int ts = tail_s;
  if (ts == 0) {  // the whole hierarchy in the single-CTA tail
    OCU_TRY(tail(true, nu1, nu2, coarse_iters, s));
    for (int c = 1; c < cycles; c++) OCU_TRY(tail(false, nu1, nu2, coarse_iters, s));
    return x ? enqueue_add_correction(x, *Lx, s) : OCU_OK;
  }
  for (int l = 0; l < ts; l++) OCU_TRY(restrict_to(l, s, true));
  OCU_TRY(tail(true, nu1, nu2, coarse_iters, s));
  for (int f = ts - 1; f >= 1; f--) {
    OCU_TRY(prolong_from(f + 1, s, CHQ_P_ASSIGN));
    OCU_TRY(relax(f, ramp_iters, false, s));
  }
  OCU_TRY(prolong_from(1, s, CHQ_P_ASSIGN));
  const int xmode = x && vec_ok(*Lx) ? CHQ_P_X64V : CHQ_P_X64;
  for (int c = 0; c < cycles; c++) {
    for (int l = 0; l < ts; l++) {
      OCU_TRY(relax(l, nu1, false, s));
      OCU_TRY(restrict_to(l, s));
    }
    OCU_TRY(tail(false, nu1, nu2, coarse_iters, s));
    for (int l = ts - 1; l >= 0; l--) {
      if (l == 0 && x && c == cycles - 1) return prolong_from(1, s, xmode, x, Lx);
      OCU_TRY(prolong_from(l + 1, s));
      if (l > 0) OCU_TRY(relax(l, nu2, false, s));
    }
  }
  return x ? enqueue_add_correction(x, *Lx, s) : OCU_OK;
}

ocu_status ChequerMG::enqueue_residual(const double *x, const double *b, const ocu_layout &L, double h, double fx_,
                                       double fy_, double fz_, double *rows2, double *rowsinf, cudaStream_t s) {
  const ChqLevel &C0 = lv[0];
  OuterCoef c;
  c.fxh = fx_ / (h * h);
  c.fyh = fy_ / (h * h);
  c.fzh = fz_ / (h * h);
  c.dg = 2 * (fx_ + fy_ + fz_) / (h * h);
  dim3 block(32, 8), grid(1, (L.ny + 7) / 8, L.nx);
  if (vec_ok(L))
    launch_pdl(k_chq_outer_residual<true>, grid, block, 0, s, x, b, (long long)L.xstride, (long long)L.ystride, L.nx,
               L.ny, L.nz, c, C0.b[0], C0.b[1], C0.rz, rows2, rowsinf);
  else
    launch_pdl(k_chq_outer_residual<false>, grid, block, 0, s, x, b, (long long)L.xstride, (long long)L.ystride, L.nx,
               L.ny, L.nz, c, C0.b[0], C0.b[1], C0.rz, rows2, rowsinf);
  return check_launch("k_chq_outer_residual");
}

ocu_status ChequerMG::enqueue_add_correction(double *x, const ocu_layout &L, cudaStream_t s) {
  const ChqLevel &C0 = lv[0];
  const int mz = (L.nz + 1) / 2;
  dim3 block(64, 4), grid((mz + 63) / 64, (L.ny + 3) / 4, L.nx);
  if (vec_ok(L))
    launch_pdl(k_chq_add_correction<true>, grid, block, 0, s, x, (long long)L.xstride, (long long)L.ystride, L.nx,
               L.ny, L.nz, C0.u[0], C0.u[1], C0.rz);
  else
    launch_pdl(k_chq_add_correction<false>, grid, block, 0, s, x, (long long)L.xstride, (long long)L.ystride, L.nx,
               L.ny, L.nz, C0.u[0], C0.u[1], C0.rz);
  return check_launch("k_chq_add_correction");
}

}  // namespace ocub
