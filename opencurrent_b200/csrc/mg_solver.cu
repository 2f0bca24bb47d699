// Multigrid pressure solver: the host-side driver of Sol_MultigridPressure3DBase /
// Sol_MultigridPressure3DDevice<T> / Sol_MultigridPressureMixed3DDeviceD, re-implemented over
// the sm_100a level kernels.  The cycle schedule (FMG ramp, convergence test after the level-0
// pre-smooth, retry with a zero initial guess) is the reference's
// (ocuequation/sol_mgpressure3d.cpp:113-398); what changed is where the work runs:
//   - every level operation is an asynchronous launch on the solver's stream (the reference
//     synchronises after every launch, ocuutil/kernel_wrapper.cu:136-167);
//   - the coarsest level is relaxed by one single-CTA kernel instead of a D2H/host/H2D round
//     trip (sol_mgpressure3ddev.cu:134-188);
//   - norms are one deterministic launch each, and the host waits only when it needs a norm
//     to decide convergence.
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "mg_solver.h"

namespace ocub {

enum { RO_RED_BLACK = 0, RO_BLACK_RED = 1, RO_SYMMETRIC = 2 };

static double min3(double a, double b, double c) { return a < b ? (a < c ? a : c) : (b < c ? b : c); }

// Sol_MultigridPressure3DBase::num_levels (sol_mgpressure3d.cpp:67-92)
int mg_num_levels(int nx_val, int ny_val, int nz_val) {
  int cnx = nx_val / 2, cny = ny_val / 2, cnz = nz_val / 2, levels = 0;
  while (2 * cnx == nx_val && 2 * cny == ny_val && 2 * cnz == nz_val) {
    levels++;
    nx_val = cnx; ny_val = cny; nz_val = cnz;
    cnx /= 2; cny /= 2; cnz /= 2;
    if (cnx < 2 || nx_val == 5 || nx_val == 7) break;
    if (cny < 2 || ny_val == 5 || ny_val == 7) break;
    if (cnz < 2 || nz_val == 5 || nz_val == 7) break;
  }
  return levels;
}

// Yavneh's red-black SOR factor (sol_mgpressure3d.cpp:94-109)
double mg_optimal_omega(double fx, double fy, double fz) {
  double f_min = min3(fx, fy, fz);
  double c_max = (1.0 - f_min / (fx + fy + fz));
  double c_max_sqr = c_max * c_max;
  return 2.0 / (1.0 + sqrt(1.0f - c_max_sqr));
}

// ------------------------------------------------------------------------------------------
// Typed level storage + operations (Sol_MultigridPressure3DDevice<T>)
// ------------------------------------------------------------------------------------------
template <typename T>
MGCore<T>::~MGCore() {
  for (size_t l = 0; l < grids_u.size(); l++) {
    if (l > 0) { if (grids_u[l]) { cudaFree(grids_u[l]->buf); delete grids_u[l]; } }
    if (l > 0 && grids_b[l]) { cudaFree(grids_b[l]->buf); delete grids_b[l]; }
    if (grids_r[l]) { cudaFree(grids_r[l]->buf); delete grids_r[l]; }
  }
  for (auto p : diag) cudaFree(p);
  if (red_scratch) cudaFree(red_scratch);
  if (d_norms) cudaFree(d_norms);
  if (h_norms) cudaFreeHost(h_norms);
}

static ocu_grid *alloc_grid(ocu_dtype dt, const ocu_layout &L, ocu_status *st) {
  ocu_grid *g = new ocu_grid;
  g->dtype = dt;
  g->L = L;
  g->owned = true;
  g->buf = nullptr;
  cudaError_t e = cudaMalloc(&g->buf, dtype_size(dt) * L.allocated);
  if (e != cudaSuccess) {
    delete g;
    *st = check_cuda(e, "cudaMalloc");
    return nullptr;
  }
  e = cudaMemset(g->buf, 0, dtype_size(dt) * L.allocated);
  if (e != cudaSuccess) { *st = check_cuda(e, "cudaMemset"); }
  return g;
}

// initialize_base_storage + initialize_storage (sol_mgpressure3d.cpp:401-437,
// sol_mgpressure3ddev.cu:376-482)
template <typename T>
ocu_status MGCore<T>::init(const ocu_bc_set &bc_, bool disable_host, int nx, int ny, int nz, double hx,
                           double hy, double hz, ocu_grid *rhs, ocu_grid *pressure, cudaStream_t s) {
  const ocu_dtype dt = sizeof(T) == 8 ? OCU_F64 : OCU_F32;
  stream = s;
  bc = bc_;
  disable_relax_on_host = disable_host;
  num_levels = mg_num_levels(nx, ny, nz);
  if (num_levels < 1)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDevice::initialize_storage - grid (%d,%d,%d) cannot be coarsened", nx, ny, nz);
  h.assign(num_levels, 0);
  dim.assign(num_levels, {0, 0, 0});
  h[0] = min3(hx, hy, hz);
  fx = (h[0] * h[0]) / (hx * hx);
  fy = (h[0] * h[0]) / (hy * hy);
  fz = (h[0] * h[0]) / (hz * hz);
  omega = mg_optimal_omega(fx, fy, fz);
  dim[0] = {nx, ny, nz};
  for (int l = 1; l < num_levels; l++) {
    h[l] = h[l - 1] * 2;
    dim[l] = {dim[l - 1][0] / 2, dim[l - 1][1] / 2, dim[l - 1][2] / 2};
  }
  update_bc_between_colors = bc_any_periodic(bc);
  lay.resize(num_levels);
  grids_u.assign(num_levels, nullptr);
  grids_b.assign(num_levels, nullptr);
  grids_r.assign(num_levels, nullptr);
  lay[0] = rhs->L;
  grids_b[0] = rhs;
  grids_u[0] = pressure;
  ocu_status st = OCU_OK;
  grids_r[0] = alloc_grid(dt, rhs->L, &st);
  if (!grids_r[0]) return st;
  for (int l = 1; l < num_levels; l++) {
    layout_compute(dim[l][0], dim[l][1], dim[l][2], 1, 1, 1, 0, 0, 0, &lay[l]);
    grids_u[l] = alloc_grid(dt, lay[l], &st);
    grids_b[l] = alloc_grid(dt, lay[l], &st);
    grids_r[l] = alloc_grid(dt, lay[l], &st);
    if (!grids_u[l] || !grids_b[l] || !grids_r[l]) return st;
  }
  if (sizeof(T) == 8) {
    diag.assign(num_levels, nullptr);
    for (int l = 0; l < num_levels; l++) {
      OCU_TRY(check_cuda(cudaMalloc(&diag[l], sizeof(T) * (size_t)dim[l][0] * dim[l][1]), "cudaMalloc(diag)"));
      RelaxParams p = relax_params(l);
      OCU_TRY(launch_init_diag<T>((T *)diag[l], dim[l][0], dim[l][1], p, stream));
    }
  }
  OCU_TRY(check_cuda(cudaMalloc(&red_scratch, reduce_scratch_bytes(lay[0], sizeof(T))), "cudaMalloc(reduce)"));
  OCU_TRY(check_cuda(cudaMemset(red_scratch, 0, reduce_scratch_bytes(lay[0], sizeof(T))), "cudaMemset(reduce)"));
  OCU_TRY(check_cuda(cudaMalloc(&d_norms, 2 * sizeof(double)), "cudaMalloc(norms)"));
  OCU_TRY(check_cuda(cudaMallocHost(&h_norms, 2 * sizeof(double)), "cudaMallocHost(norms)"));
  return check_cuda(cudaStreamSynchronize(stream), "initialize_storage");
}

template <typename T>
ocu_bc_set MGCore<T>::bc_at_level(int level) const {
  ocu_bc_set b = bc;
  if (level != 0) bc_make_homogeneous(&b);
  return b;
}

template <typename T>
RelaxParams MGCore<T>::relax_params(int level) const {
  RelaxParams p;
  p.omega = omega;
  p.h = h[level];
  p.fx = fx; p.fy = fy; p.fz = fz;
  p.bc = bc_at_level(level);
  return p;
}

template <typename T>
ocu_status MGCore<T>::apply_bc(int level) {
  return launch_bc_level1<T>(u0(level), lay[level], bc_at_level(level), hx(level), hy(level), hz(level), stream);
}

template <typename T>
ocu_status MGCore<T>::clear_zero(int level) {
  return check_cuda(cudaMemsetAsync(grids_u[level]->buf, 0, sizeof(T) * lay[level].allocated, stream), "clear_zero");
}

// relax (sol_mgpressure3ddev.cu:190-248)
template <typename T>
ocu_status MGCore<T>::relax(int level, int iterations, int order) {
  const RelaxParams p = relax_params(level);
  if (!disable_relax_on_host && level == num_levels - 1)
    return launch_coarse_relax<T>(u0(level), b0(level), lay[level], iterations, order, p, hx(level), hy(level),
                                  hz(level), stream);
  if (order == RO_SYMMETRIC) {
    if (iterations % 2 == 1) iterations++;
    if (iterations < 4) iterations = 4;
  }
  const T *dg = diag.empty() ? nullptr : (const T *)diag[level];
  for (int it = 0; it < iterations; it++) {
    for (int rb = 0; rb < 2; rb++) {
      int color = rb;
      if (order == RO_BLACK_RED || (order == RO_SYMMETRIC && it >= iterations / 2)) color = !rb;
      OCU_TRY(launch_relax_color<T>(u0(level), b0(level), lay[level], dg, color, p, stream));
      if (update_bc_between_colors) OCU_TRY(apply_bc(level));
    }
    if (!update_bc_between_colors) OCU_TRY(apply_bc(level));
  }
  return OCU_OK;
}

// restrict_residuals (sol_mgpressure3ddev.cu:250-279): the squared-residual sum is folded in
// T, divided by the cell count in T and square-rooted in T.
template <typename T>
ocu_status MGCore<T>::restrict_residuals(int fine, int coarse, double *l2, double *linf) {
  const double hf = h[fine];
  OCU_TRY(launch_residual<T>(u0(fine), b0(fine), r0(fine), lay[fine], hf, fx, fy, fz, stream));
  if (coarse != fine) OCU_TRY(launch_restrict<T>(r0(fine), lay[fine], b0(coarse), lay[coarse], stream));
  if (l2 || linf) {
    if (l2) OCU_TRY(launch_reduce<T>(r0(fine), lay[fine], OCU_REDUCE_SQRSUM, red_scratch, d_norms, stream));
    if (linf) OCU_TRY(launch_reduce<T>(r0(fine), lay[fine], OCU_REDUCE_MAXABS, red_scratch, d_norms + 1, stream));
    OCU_TRY(check_cuda(cudaMemcpyAsync(h_norms, d_norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream),
                       "norm readback"));
    OCU_TRY(check_cuda(cudaStreamSynchronize(stream), "norm readback"));
    if (l2) {
      T rn = (T)h_norms[0];
      rn /= (T)(dim[fine][0] * dim[fine][1] * dim[fine][2]);
      *l2 = (double)std::sqrt(rn);
    }
    if (linf) *linf = h_norms[1];
  }
  return OCU_OK;
}

// prolong (sol_mgpressure3ddev.cu:284-297)
template <typename T>
ocu_status MGCore<T>::prolong(int coarse, int fine) {
  OCU_TRY(launch_prolong<T>(u0(coarse), lay[coarse], u0(fine), lay[fine], stream));
  return apply_bc(fine);
}

template struct MGCore<float>;
template struct MGCore<double>;

// ------------------------------------------------------------------------------------------
// Driver (Sol_MultigridPressure3DBase)
// ------------------------------------------------------------------------------------------
CoreOps *MGSolver::active() { return double_mode ? (CoreOps *)&cd : (CoreOps *)&cf; }

int MGSolver::coarse_iters() const {
  const int cl = num_levels - 1;
  const auto &d = (kind == OCU_MG_F32) ? cf.dim[cl] : cd.dim[cl];
  const int a = d[0] * d[1], b = d[1] * d[2], c = d[0] * d[2];
  const int mx = a > b ? (a > c ? a : c) : (b > c ? b : c);
  return mx / 2;
}

static double pick(int conv, double l2, double linf) {
  return (conv & OCU_CONVERGENCE_CRITERIA_L2) ? l2 : (conv & OCU_CONVERGENCE_CRITERIA_LINF) ? linf : 1e20;
}

// do_fmg (sol_mgpressure3d.cpp:113-251); returns OCU_OK (converged), OCU_ERR_NOT_CONVERGED, or
// an error.
ocu_status MGSolver::do_fmg(double tolerance, int max_iter, double *rl2, double *rlinf) {
  const int conv = prm.convergence;
  const int coarse_level = num_levels - 1;
  int num_vcyc = 0;
  double orig_l2 = 0, orig_linf = 0;
  *rl2 = *rlinf = 0;
  CoreOps *c = active();
  OCU_TRY(c->apply_bc(0));
  OCU_TRY(c->restrict_residuals(0, 0, (conv & OCU_CONVERGENCE_CALC_L2) ? &orig_l2 : nullptr,
                                (conv & OCU_CONVERGENCE_CALC_LINF) ? &orig_linf : nullptr));
  if (pick(conv, orig_l2, orig_linf) < tolerance) {
    if (conv & OCU_CONVERGENCE_CALC_L2) *rl2 = orig_l2;
    if (conv & OCU_CONVERGENCE_CALC_LINF) *rlinf = orig_linf;
    stats.vcycles = 0;
    return OCU_OK;
  }
  for (int level = 0; level < num_levels - 1; level++) {
    OCU_TRY(c->clear_zero(level + 1));
    OCU_TRY(c->apply_bc(level + 1));
    OCU_TRY(c->restrict_residuals(level, level + 1, nullptr, nullptr));
  }
  for (int fine_level = num_levels - 1; fine_level >= 0; fine_level--) {
    const int level_ncyc = (fine_level == 0) ? max_iter + 1 : 1;
    for (int i_cyc = 0; i_cyc < level_ncyc; i_cyc++) {
      if (fine_level == 0) num_vcyc++;
      for (int level = fine_level; level < coarse_level; level++) {
        OCU_TRY(c->relax(level, prm.nu1, RO_RED_BLACK));
        OCU_TRY(c->clear_zero(level + 1));
        OCU_TRY(c->apply_bc(level + 1));
        if (level == 0) {
          OCU_TRY(c->restrict_residuals(0, 1, (conv & OCU_CONVERGENCE_CALC_L2) ? rl2 : nullptr,
                                        (conv & OCU_CONVERGENCE_CALC_LINF) ? rlinf : nullptr));
          stats.last_l2 = *rl2;
          stats.last_linf = *rlinf;
          if (pick(conv, *rl2, *rlinf) < tolerance) {
            OCU_TRY(c->apply_bc(0));
            stats.vcycles = num_vcyc;
            return OCU_OK;
          }
        } else {
          OCU_TRY(c->restrict_residuals(level, level + 1, nullptr, nullptr));
        }
      }
      OCU_TRY(c->relax(coarse_level, coarse_iters(), prm.make_symmetric_operator ? RO_SYMMETRIC : RO_RED_BLACK));
      for (int level = coarse_level - 1; level >= fine_level; level--) {
        OCU_TRY(c->prolong(level + 1, level));
        if (level > 0)
          OCU_TRY(c->relax(level, prm.nu2, prm.make_symmetric_operator ? RO_BLACK_RED : RO_RED_BLACK));
      }
    }
    if (fine_level > 0) OCU_TRY(c->prolong(fine_level, fine_level - 1));
  }
  stats.vcycles = num_vcyc;
  return OCU_ERR_NOT_CONVERGED;
}

// do_vcycle (sol_mgpressure3d.cpp:253-329)
ocu_status MGSolver::do_vcycle(double tolerance, int max_iter, double *rl2, double *rlinf) {
  const int conv = prm.convergence;
  const int coarse_level = num_levels - 1;
  double orig_l2 = 0, orig_linf = 0;
  CoreOps *c = active();
  OCU_TRY(c->apply_bc(0));
  OCU_TRY(c->restrict_residuals(0, 0, (conv & OCU_CONVERGENCE_CALC_L2) ? &orig_l2 : nullptr,
                                (conv & OCU_CONVERGENCE_CALC_LINF) ? &orig_linf : nullptr));
  if (pick(conv, orig_l2, orig_linf) < tolerance) {
    if (conv & OCU_CONVERGENCE_CALC_L2) *rl2 = orig_l2;
    if (conv & OCU_CONVERGENCE_CALC_LINF) *rlinf = orig_linf;
    return OCU_OK;
  }
  for (int i_cyc = 0; i_cyc < max_iter; i_cyc++) {
    for (int level = 0; level < coarse_level; level++) {
      OCU_TRY(c->relax(level, prm.nu1, RO_RED_BLACK));
      OCU_TRY(c->clear_zero(level + 1));
      OCU_TRY(c->apply_bc(level + 1));
      if (level == 0) {
        OCU_TRY(c->restrict_residuals(0, 1, (conv & OCU_CONVERGENCE_CALC_L2) ? rl2 : nullptr,
                                      (conv & OCU_CONVERGENCE_CALC_LINF) ? rlinf : nullptr));
        if (pick(conv, *rl2, *rlinf) < tolerance) {
          OCU_TRY(c->apply_bc(0));
          return OCU_OK;
        }
      } else {
        OCU_TRY(c->restrict_residuals(level, level + 1, nullptr, nullptr));
      }
    }
    OCU_TRY(c->relax(coarse_level, coarse_iters(), prm.make_symmetric_operator ? RO_SYMMETRIC : RO_RED_BLACK));
    for (int level = coarse_level - 1; level >= 0; level--) {
      OCU_TRY(c->prolong(level + 1, level));
      if (level > 0)
        OCU_TRY(c->relax(level, prm.nu2, prm.make_symmetric_operator ? RO_BLACK_RED : RO_RED_BLACK));
    }
  }
  return OCU_ERR_NOT_CONVERGED;
}

// Sol_MultigridPressureMixed3DDeviceD::do_fmg (sol_mgpressuremixed3ddevd.cpp:79-100)
ocu_status MGSolver::mixed_warmstart_fmg(double tolerance, int max_iter, double *rl2, double *rlinf) {
  const ocu_layout &L = cd.lay[0];
  OCU_TRY(launch_convert<float, double>((float *)rhs_f->buf, (const double *)cd.grids_b[0]->buf, L.allocated, stream));
  double_mode = false;
  ocu_status st = do_fmg(tolerance > 1e-2 ? tolerance : 1e-2, 4, rl2, rlinf);
  if (st != OCU_OK && st != OCU_ERR_NOT_CONVERGED) return st;
  OCU_TRY(launch_convert<double, float>((double *)cd.grids_u[0]->buf, (const float *)cf.grids_u[0]->buf,
                                        L.allocated, stream));
  double_mode = true;
  if (tolerance < 1e-2 || prm.convergence == OCU_CONVERGENCE_L2) {
    st = do_fmg(tolerance, max_iter, rl2, rlinf);
    OCU_TRY(launch_convert<float, double>((float *)cf.grids_u[0]->buf, (const double *)cd.grids_u[0]->buf,
                                          L.allocated, stream));
    return st;
  }
  return OCU_OK;
}

// FP32-in-FP64 iterative refinement.  Outer loop in FP64: r = b - A x (residual kernel + norm
// folds in double), stop when the norm is below tolerance; otherwise solve A e = (float) r with
// a fixed FP32 FMG schedule (ir_inner_cycles fine-level cycles, homogeneous boundary values)
// and update x += (double) e.  max_outer bounds the refinement steps.
ocu_status MGSolver::ir_solve(double tolerance, int max_outer, double *rl2, double *rlinf) {
  const int conv = prm.convergence;
  const ocu_layout &L = cd.lay[0];
  double l2 = 0, linf = 0;
  stats.outer_iterations = 0;
  stats.vcycles = 0;
  double_mode = true;
  OCU_TRY(cd.apply_bc(0));
  OCU_TRY(cd.restrict_residuals(0, 0, &l2, &linf));
  *rl2 = l2; *rlinf = linf;
  stats.last_l2 = l2; stats.last_linf = linf;
  if (pick(conv, l2, linf) < tolerance) return OCU_OK;
  const int inner = prm.ir_inner_cycles > 0 ? prm.ir_inner_cycles : 3;
  ocu_mg_params saved = prm;
  int total_inner = 0;
  for (int outer = 1; outer <= max_outer; outer++) {
    OCU_TRY(launch_downcast_interior((const double *)cd.r0(0), (float *)cf.b0(0), L, stream));
    OCU_TRY(cf.clear_zero(0));
    prm.convergence = OCU_CONVERGENCE_NONE;
    double_mode = false;
    double el2, elinf;
    ocu_status st = do_fmg(0.0, inner - 1, &el2, &elinf);
    total_inner += stats.vcycles;
    prm = saved;
    double_mode = true;
    if (st != OCU_OK && st != OCU_ERR_NOT_CONVERGED) return st;
    OCU_TRY(launch_add_correction((double *)cd.u0(0), (const float *)cf.u0(0), L, stream));
    OCU_TRY(cd.apply_bc(0));
    OCU_TRY(cd.restrict_residuals(0, 0, &l2, &linf));
    stats.outer_iterations = outer;
    stats.vcycles = total_inner;
    *rl2 = l2; *rlinf = linf;
    stats.last_l2 = l2; stats.last_linf = linf;
    if (pick(conv, l2, linf) < tolerance) return OCU_OK;
  }
  return OCU_ERR_NOT_CONVERGED;
}

ocu_status MGSolver::fmg_dispatch(double tol, int max_iter, double *l2, double *linf) {
  if (kind == OCU_MG_MIXED_WARMSTART) return mixed_warmstart_fmg(tol, max_iter, l2, linf);
  if (kind == OCU_MG_MIXED_IR) return ir_solve(tol, max_iter, l2, linf);
  return do_fmg(tol, max_iter, l2, linf);
}

// Base::solve (sol_mgpressure3d.cpp:332-370)
ocu_status MGSolver::solve(double *residual, double tolerance, int max_iter) {
  if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] Sol_MultigridPressure3DDevice::solve - not initialized");
  if (!check_float((float)tolerance))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDevice::solve - garbage tolerance value %f", tolerance);
  if (tolerance < 0)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDevice::solve - negative tolerance value %f", tolerance);
  if (max_iter <= 0)
    return fail(OCU_ERR_INVALID_VALUE, "[WARNING] Sol_MultigridPressure3DDevice::solve - non-positive max_iter %d", max_iter);
  double l2 = 0, linf = 0;
  ocu_status st = fmg_dispatch(tolerance, max_iter, &l2, &linf);
  if (st == OCU_ERR_NOT_CONVERGED) {
    // retry with a zeroed initial guess (sol_mgpressure3d.cpp:351-364)
    OCU_TRY(active()->clear_zero(0));
    st = fmg_dispatch(tolerance, max_iter, &l2, &linf);
  }
  *residual = (prm.convergence == OCU_CONVERGENCE_L2) ? l2 : linf;
  stats.last_l2 = l2;
  stats.last_linf = linf;
  if (st == OCU_ERR_NOT_CONVERGED)
    set_error("[WARNING] Sol_MultigridPressure3DBase::solve - do_fmg failed, residual %g", *residual);
  return st;
}

ocu_status MGSolver::run_vcycles(int count) {
  if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] run_vcycles - not initialized");
  if (count <= 0) return fail(OCU_ERR_INVALID_VALUE, "[WARNING] Sol_MultigridPressure3DDevice::run_vcycles - non-positive count %d", count);
  double l2, linf;
  ocu_status st = do_vcycle(0, count, &l2, &linf);
  if (st == OCU_ERR_NOT_CONVERGED) st = OCU_OK;
  if (st == OCU_OK) st = check_cuda(cudaStreamSynchronize(stream), "run_vcycles");
  return st;
}

ocu_status MGSolver::run_fmg(int count) {
  if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] run_fmg - not initialized");
  if (count < 0) return fail(OCU_ERR_INVALID_VALUE, "[WARNING] Sol_MultigridPressure3DDevice::run_fmg - negative count %d", count);
  double l2, linf;
  ocu_status st = do_fmg(0, count, &l2, &linf);
  if (st == OCU_ERR_NOT_CONVERGED) st = OCU_OK;
  if (st == OCU_OK) st = check_cuda(cudaStreamSynchronize(stream), "run_fmg");
  return st;
}

MGSolver::~MGSolver() {
  if (pressure) { cudaFree(pressure->buf); delete pressure; }
  if (rhs_f) { cudaFree(rhs_f->buf); delete rhs_f; }
}

ocu_status MGSolver::initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, ocu_grid *rhs) {
  if (initialized) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] initialize_storage - already initialized");
  if (!check_float((float)hx) || !check_float((float)hy) || !check_float((float)hz))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DBase::initialize_storage - garbage hx,hy,hz value %f %f %f", hx, hy, hz);
  if (!rhs) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] initialize_storage - null rhs");
  const ocu_dtype want = (kind == OCU_MG_F32) ? OCU_F32 : OCU_F64;
  if (rhs->dtype != want) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] initialize_storage - rhs element type mismatch");
  if (rhs->L.gx < 1 || rhs->L.gy < 1 || rhs->L.gz < 1)
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_MultigridPressure3DDevice::initialize_storage - rhs has invalid ghost cells (%d,%d,%d), must be >= 1", rhs->L.gx, rhs->L.gy, rhs->L.gz);
  if (rhs->L.nx != nx || rhs->L.ny != ny || rhs->L.nz != nz)
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_MultigridPressure3DDevice::initialize_storage - rhs dimension mismatch (%d,%d,%d) != (%d,%d,%d)", rhs->L.nx, rhs->L.ny, rhs->L.nz, nx, ny, nz);
  ocu_status st = OCU_OK;
  pressure = alloc_grid(want, rhs->L, &st);
  if (!pressure) return st;
  const bool dis = prm.disable_relax_on_host != 0;
  if (kind == OCU_MG_F32) {
    OCU_TRY(cf.init(prm.bc, dis, nx, ny, nz, hx, hy, hz, rhs, pressure, stream));
    num_levels = cf.num_levels;
    double_mode = false;
    stats.omega = cf.omega;
  } else {
    OCU_TRY(cd.init(prm.bc, dis, nx, ny, nz, hx, hy, hz, rhs, pressure, stream));
    num_levels = cd.num_levels;
    double_mode = true;
    stats.omega = cd.omega;
    if (kind == OCU_MG_MIXED_WARMSTART || kind == OCU_MG_MIXED_IR) {
      rhs_f = alloc_grid(OCU_F32, rhs->L, &st);
      if (!rhs_f) return st;
      ocu_grid *pf = alloc_grid(OCU_F32, rhs->L, &st);
      if (!pf) return st;
      pressure_f.reset(pf);
      ocu_bc_set fbc = prm.bc;
      if (kind == OCU_MG_MIXED_IR) bc_make_homogeneous(&fbc);
      OCU_TRY(cf.init(fbc, dis, nx, ny, nz, hx, hy, hz, rhs_f, pf, stream));
    }
  }
  stats.num_levels = num_levels;
  initialized = true;
  return OCU_OK;
}

ocu_status MGSolver::set_params(const ocu_mg_params &p) {
  prm = p;
  cf.bc = p.bc;
  cd.bc = p.bc;
  if (kind == OCU_MG_MIXED_IR) bc_make_homogeneous(&cf.bc);
  cf.disable_relax_on_host = cd.disable_relax_on_host = p.disable_relax_on_host != 0;
  return OCU_OK;
}

void MGSolver::set_stream(cudaStream_t s) {
  stream = s;
  cf.stream = s;
  cd.stream = s;
}

ocu_grid *MGSolver::level_grid(char which, int level) {
  if (!initialized || level < 0 || level >= num_levels) return nullptr;
  auto &core = (kind == OCU_MG_F32) ? (CoreOps &)cf : (CoreOps &)cd;
  return core.grid(which, level);
}

}  // namespace ocub
