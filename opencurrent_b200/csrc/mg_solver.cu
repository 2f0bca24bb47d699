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

#include "ghost_emit.cuh"
#include "mg_fused.h"
#include "mg_solver.h"

namespace ocub {


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
  for (auto g : grids_u2)
    if (g) { cudaFree(g->buf); delete g; }
  for (auto p : diag) cudaFree(p);
  if (red_scratch) cudaFree(red_scratch);
  if (rows) cudaFree(rows);
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
ocu_status MGCore<T>::set_geometry(const ocu_bc_set &bc_, bool disable_host, int nx, int ny, int nz, double hx,
                                   double hy, double hz, const ocu_layout &L0) {
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
  lay[0] = L0;
  for (int l = 1; l < num_levels; l++) layout_compute(dim[l][0], dim[l][1], dim[l][2], 1, 1, 1, 0, 0, 0, &lay[l]);
  return OCU_OK;
}

template <typename T>
ocu_status MGCore<T>::init(const ocu_bc_set &bc_, bool disable_host, int nx, int ny, int nz, double hx,
                           double hy, double hz, ocu_grid *rhs, ocu_grid *pressure, cudaStream_t s) {
  const ocu_dtype dt = sizeof(T) == 8 ? OCU_F64 : OCU_F32;
  stream = s;
  OCU_TRY(set_geometry(bc_, disable_host, nx, ny, nz, hx, hy, hz, rhs->L));
  grids_u.assign(num_levels, nullptr);
  grids_b.assign(num_levels, nullptr);
  grids_r.assign(num_levels, nullptr);
  grids_b[0] = rhs;
  grids_u[0] = pressure;
  ocu_status st = OCU_OK;
  grids_r[0] = alloc_grid(dt, rhs->L, &st);
  if (!grids_r[0]) return st;
  for (int l = 1; l < num_levels; l++) {
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
  rows_stride = ((long long)dim[0][0] * dim[0][1] + 63) / 64 * 64;
  OCU_TRY(check_cuda(cudaMalloc(&rows, 2 * sizeof(T) * rows_stride), "cudaMalloc(norm rows)"));
  // norms[0..1] = l2, linf; norms[2] holds the kernels' timeout word (read back with the norms)
  OCU_TRY(check_cuda(cudaMalloc(&d_norms, 4 * sizeof(double)), "cudaMalloc(norms)"));
  OCU_TRY(check_cuda(cudaMemset(d_norms, 0, 4 * sizeof(double)), "cudaMemset(norms)"));
  OCU_TRY(check_cuda(cudaMallocHost(&h_norms, 4 * sizeof(double)), "cudaMallocHost(norms)"));
  std::memset(h_norms, 0, 4 * sizeof(double));
  d_err = reinterpret_cast<int *>(d_norms + 2);
  grids_u2.assign(num_levels, nullptr);
  tm_u.resize(num_levels);
  tm_u2.resize(num_levels);
  tm_b.resize(num_levels);
  return check_cuda(cudaStreamSynchronize(stream), "initialize_storage");
}

// Second u buffer + TMA maps for every level the two-colour pass may run on; allocated when the
// pass is first enabled (never inside a stream capture: set_params / initialize_storage only).
template <typename T>
ocu_status MGCore<T>::ensure_sweep_buffers() {
  const ocu_dtype dt = sizeof(T) == 8 ? OCU_F64 : OCU_F32;
  ocu_status st = OCU_OK;
  for (int l = 0; l < num_levels; l++) {
    if (grids_u2[l] || !sweep2_supported(lay[l], bc_at_level(l))) continue;
    if ((long long)dim[l][0] * dim[l][1] * dim[l][2] < 512) continue;
    grids_u2[l] = alloc_grid(dt, lay[l], &st);
    if (!grids_u2[l]) return st;
    OCU_TRY(make_sweep_tmap<T>(grids_u[l]->buf, lay[l], &tm_u[l]));
    OCU_TRY(make_sweep_tmap<T>(grids_u2[l]->buf, lay[l], &tm_u2[l]));
    OCU_TRY(make_sweep_tmap<T>(grids_b[l]->buf, lay[l], &tm_b[l]));
  }
  return OCU_OK;
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
  // a kernel rather than a memset node, so that the launches around it keep their programmatic
  // (overlapped) dependencies
  return launch_clear<T>(static_cast<T *>(grids_u[level]->buf), lay[level].allocated, (T)0, stream);
}

// clear_zero(level) followed by apply_boundary_conditions(level).  Below level 0 the boundary
// values are homogeneous, so every ghost rule maps the zero interior to +0 -- the same bits the
// memset wrote -- and the ghost launch is skipped.
template <typename T>
ocu_status MGCore<T>::clear_level(int level) {
  OCU_TRY(clear_zero(level));
  return level == 0 ? apply_bc(level) : OCU_OK;
}

// Ghost writes can ride along with the kernels that update interior cells when no face is
// BC_NONE and every periodic axis has an even cell count (otherwise a colour sweep would read
// a ghost written in the same sweep).
template <typename T>
bool MGCore<T>::emit_ok(int level) const {
  if (!fused) return false;
  const ocu_bc_set b = bc_at_level(level);
  if (bc_has_none(b)) return false;
  if ((b.xpos.type == OCU_BC_PERIODIC || b.xneg.type == OCU_BC_PERIODIC) && (dim[level][0] & 1)) return false;
  if ((b.ypos.type == OCU_BC_PERIODIC || b.yneg.type == OCU_BC_PERIODIC) && (dim[level][1] & 1)) return false;
  if ((b.zpos.type == OCU_BC_PERIODIC || b.zneg.type == OCU_BC_PERIODIC) && (dim[level][2] & 1)) return false;
  return true;
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
  const bool emit = emit_ok(level);
  if (emit && sweep2_ok(level)) return relax_pairs(level, iterations, order);
  for (int it = 0; it < iterations; it++) {
    for (int rb = 0; rb < 2; rb++) {
      int color = rb;
      if (order == RO_BLACK_RED || (order == RO_SYMMETRIC && it >= iterations / 2)) color = !rb;
      if (emit) {
        OCU_TRY(launch_relax_color_emit<T>(u0(level), b0(level), lay[level], dg, color, p, hx(level), hy(level),
                                           hz(level), stream));
      } else {
        OCU_TRY(launch_relax_color<T>(u0(level), b0(level), lay[level], dg, color, p, stream));
        if (update_bc_between_colors) OCU_TRY(apply_bc(level));
      }
    }
    if (!emit && !update_bc_between_colors) OCU_TRY(apply_bc(level));
  }
  return OCU_OK;
}

template <typename T>
bool MGCore<T>::sweep2_ok(int level) const {
  if (!fused || sweep_cells <= 0 || level >= (int)grids_u2.size() || !grids_u2[level]) return false;
  if (!sweep2_supported(lay[level], bc_at_level(level))) return false;  // the BCs may have changed
  return (long long)dim[level][0] * dim[level][1] * dim[level][2] >= sweep_cells;
}

// Iterations in pairs through the two-colour pass (u -> u2 -> u, so the result stays in u);
// an odd last iteration runs as two colour launches.  Same colour order as relax().
template <typename T>
ocu_status MGCore<T>::relax_pairs(int level, int iterations, int order) {
  const RelaxParams p = relax_params(level);
  const T *dg = diag.empty() ? nullptr : (const T *)diag[level];
  auto first = [&](int it) {
    return (order == RO_BLACK_RED || (order == RO_SYMMETRIC && it >= iterations / 2)) ? 1 : 0;
  };
  int it = 0;
  for (; it + 1 < iterations; it += 2) {
    OCU_TRY(launch_relax_sweep2<T>(tm_u[level], tm_b[level], origin<T>(grids_u2[level]), lay[level], dg, first(it), p,
                                   hx(level), hy(level), hz(level), d_err, stream, wait_limit));
    OCU_TRY(launch_relax_sweep2<T>(tm_u2[level], tm_b[level], u0(level), lay[level], dg, first(it + 1), p, hx(level),
                                   hy(level), hz(level), d_err, stream, wait_limit));
  }
  for (; it < iterations; it++)
    for (int rb = 0; rb < 2; rb++)
      OCU_TRY(launch_relax_color_emit<T>(u0(level), b0(level), lay[level], dg, first(it) ? !rb : rb, p, hx(level),
                                         hy(level), hz(level), stream));
  return OCU_OK;
}

// restrict_residuals, enqueue part (sol_mgpressure3ddev.cu:250-279).  The fused path computes
// the residual, the restriction and the norm partials in one pass without storing r; with
// store_residuals the reference's separate kernels run and r_grid(level) is kept.  Requested
// norms are folded on the device and copied to pinned host memory; finish_norms() waits.
template <typename T>
ocu_status MGCore<T>::enqueue_restrict_residuals(int fine, int coarse, bool want_l2, bool want_linf) {
  const double hf = h[fine];
  const bool norms = want_l2 || want_linf;
  if (!fused || store_residuals) {
    OCU_TRY(launch_residual<T>(u0(fine), b0(fine), r0(fine), lay[fine], hf, fx, fy, fz, stream));
    if (coarse != fine) OCU_TRY(launch_restrict<T>(r0(fine), lay[fine], b0(coarse), lay[coarse], stream));
    if (want_l2) OCU_TRY(launch_reduce<T>(r0(fine), lay[fine], OCU_REDUCE_SQRSUM, red_scratch, d_norms, stream));
    if (want_linf) OCU_TRY(launch_reduce<T>(r0(fine), lay[fine], OCU_REDUCE_MAXABS, red_scratch, d_norms + 1, stream));
  } else {
    T *rows2 = want_l2 ? (T *)rows : nullptr;
    T *rowsinf = want_linf ? (T *)rows + rows_stride : nullptr;
    if (coarse != fine) {
      OCU_TRY(launch_residual_restrict<T>(u0(fine), b0(fine), lay[fine], b0(coarse), lay[coarse], hf, fx, fy, fz,
                                          rows2, rowsinf, stream));
    } else if (norms) {
      OCU_TRY(launch_residual_rows<T>(u0(fine), b0(fine), nullptr, nullptr, lay[fine], hf, fx, fy, fz, rows2, rowsinf,
                                      stream));
    }
    const long long nrows = (long long)dim[fine][0] * dim[fine][1];
    if (want_l2) OCU_TRY(launch_fold_rows<T>(rows2, nrows, false, red_scratch, d_norms, stream));
    if (want_linf) OCU_TRY(launch_fold_rows<T>(rowsinf, nrows, true, red_scratch, d_norms + 1, stream));
  }
  if (norms)
    OCU_TRY(launch_readback(d_norms, h_norms, 3, stream));
  return OCU_OK;
}

// clear_level(fine + 1) then the restriction into it.  On the fused path the clear (the whole
// buffer of the coarser level, the memset it stands for) rides in the restriction kernel: one
// launch less per level and cycle.
template <typename T>
ocu_status MGCore<T>::clear_and_restrict(int fine, bool want_l2, bool want_linf) {
  const int coarse = fine + 1;
  if (!fused || store_residuals) {
    OCU_TRY(clear_level(coarse));
    return enqueue_restrict_residuals(fine, coarse, want_l2, want_linf);
  }
  const bool norms = want_l2 || want_linf;
  T *rows2 = want_l2 ? (T *)rows : nullptr;
  T *rowsinf = want_linf ? (T *)rows + rows_stride : nullptr;
  OCU_TRY(launch_residual_restrict<T>(u0(fine), b0(fine), lay[fine], b0(coarse), lay[coarse], h[fine], fx, fy, fz,
                                      rows2, rowsinf, stream, static_cast<T *>(grids_u[coarse]->buf),
                                      lay[coarse].allocated));
  const long long nrows = (long long)dim[fine][0] * dim[fine][1];
  if (want_l2) OCU_TRY(launch_fold_rows<T>(rows2, nrows, false, red_scratch, d_norms, stream));
  if (want_linf) OCU_TRY(launch_fold_rows<T>(rowsinf, nrows, true, red_scratch, d_norms + 1, stream));
  if (norms)
    OCU_TRY(launch_readback(d_norms, h_norms, 3, stream));
  return OCU_OK;
}

// The squared-residual sum is folded in T, divided by the cell count in T and square-rooted in
// T (sol_mgpressure3ddev.cu:263-268).
template <typename T>
ocu_status MGCore<T>::finish_norms(int fine, double *l2, double *linf) {
  OCU_TRY(check_cuda(cudaStreamSynchronize(stream), "norm readback"));
  if (*reinterpret_cast<const int *>(h_norms + 2) != 0) {
    cudaMemsetAsync(d_err, 0, sizeof(int), stream);
    *reinterpret_cast<int *>(h_norms + 2) = 0;
    return fail(OCU_ERR_TIMEOUT, "[ERROR] multigrid - a kernel's bounded wait for its TMA loads gave up");
  }
  if (l2) {
    T rn = (T)h_norms[0];
    rn /= (T)(dim[fine][0] * dim[fine][1] * dim[fine][2]);
    *l2 = (double)std::sqrt(rn);
  }
  if (linf) *linf = h_norms[1];
  return OCU_OK;
}

template <typename T>
ocu_status MGCore<T>::restrict_residuals(int fine, int coarse, double *l2, double *linf) {
  OCU_TRY(enqueue_restrict_residuals(fine, coarse, l2 != nullptr, linf != nullptr));
  if (l2 || linf) return finish_norms(fine, l2, linf);
  return OCU_OK;
}

// prolong (sol_mgpressure3ddev.cu:284-297)
template <typename T>
ocu_status MGCore<T>::prolong(int coarse, int fine) {
  if (emit_ok(fine))
    return launch_prolong_emit<T>(u0(coarse), lay[coarse], u0(fine), lay[fine], bc_at_level(fine), hx(fine), hy(fine),
                                  hz(fine), stream);
  OCU_TRY(launch_prolong<T>(u0(coarse), lay[coarse], u0(fine), lay[fine], stream));
  return apply_bc(fine);
}

// First level handled by the single-CTA tail: the finest level >= 1 from which every level has
// at most tail_cells cells.  num_levels-1 means "coarsest only" (the plain coarse kernel).
template <typename T>
int MGCore<T>::tail_start() const {
  const int coarse = num_levels - 1;
  if (!fused || tail_cells <= 0) return coarse;
  int s = coarse;
  while (s - 1 >= 1 && (long long)dim[s - 1][0] * dim[s - 1][1] * dim[s - 1][2] <= tail_cells &&
         coarse - (s - 1) + 1 <= kMaxTailLevels)
    s--;
  return s;
}

// Tail schedule parameters for levels s..L-1 on the given level origins.
template <typename T>
void MGCore<T>::fill_tail_params(TailParams<T> &P, int s, int nu1, int nu2, int coarse_iters, bool symmetric,
                                 T *const *u_origin, T *const *b_origin) const {
  const int coarse = num_levels - 1;
  std::memset(&P, 0, sizeof(P));
  P.nlev = coarse - s + 1;
  P.first_level = s;
  P.nu1 = nu1;
  P.nu2 = nu2;
  P.post_order = symmetric ? RO_BLACK_RED : RO_RED_BLACK;
  P.host_coarse = disable_relax_on_host ? 0 : 1;
  P.coarse_order = symmetric ? RO_SYMMETRIC : RO_RED_BLACK;
  int ci = coarse_iters;
  if (P.host_coarse && P.coarse_order == RO_SYMMETRIC) {
    if (ci % 2 == 1) ci++;
    if (ci < 4) ci = 4;
  }
  P.coarse_iters = ci;
  P.cc = make_coarse_coef<T>(relax_params(coarse));
  for (int l = s; l <= coarse; l++) {
    TailLevel<T> &v = P.lv[l - s];
    v.u = u_origin[l];
    v.b = b_origin[l];
    v.xs = lay[l].xstride;
    v.ys = lay[l].ystride;
    v.nx = dim[l][0]; v.ny = dim[l][1]; v.nz = dim[l][2];
    v.emit_ok = emit_ok(l) ? 1 : 0;
    v.periodic = bc_any_periodic(bc) ? 1 : 0;
    v.bc = to_dev(bc_at_level(l));
    v.hx = (T)hx(l); v.hy = (T)hy(l); v.hz = (T)hz(l);
    v.rc = make_relax_coef_d<T>(relax_params(l));
    const double hh = h[l];
    v.res.fxh = (T)(fx / (hh * hh));
    v.res.fyh = (T)(fy / (hh * hh));
    v.res.fzh = (T)(fz / (hh * hh));
    v.res.dg = (T)(2 * (fx + fy + fz) / (hh * hh));
  }
}

// Levels s..L-1 of a V-cycle: down (relax nu1, clear, residual+restrict), coarsest relax,
// up (prolong + ghosts, relax nu2 where the absolute level is > 0).
template <typename T>
ocu_status MGCore<T>::cycle_tail(int s, int nu1, int nu2, int coarse_iters, bool symmetric) {
  const int coarse = num_levels - 1;
  if (s >= coarse) return relax(coarse, coarse_iters, symmetric ? RO_SYMMETRIC : RO_RED_BLACK);
  for (int l = s; l <= coarse; l++)
    if (!emit_ok(l) && l != coarse) {
      // ghost writes cannot be fused on this hierarchy: run the per-level kernels
      for (int q = s; q < coarse; q++) {
        OCU_TRY(relax(q, nu1, RO_RED_BLACK));
        OCU_TRY(clear_level(q + 1));
        OCU_TRY(enqueue_restrict_residuals(q, q + 1, false, false));
      }
      OCU_TRY(relax(coarse, coarse_iters, symmetric ? RO_SYMMETRIC : RO_RED_BLACK));
      for (int q = coarse - 1; q >= s; q--) {
        OCU_TRY(prolong(q + 1, q));
        if (q > 0) OCU_TRY(relax(q, nu2, symmetric ? RO_BLACK_RED : RO_RED_BLACK));
      }
      return OCU_OK;
    }
  TailParams<T> P;
  std::vector<T *> uo(num_levels), bo(num_levels);
  for (int l = 0; l < num_levels; l++) {
    uo[l] = u0(l);
    bo[l] = b0(l);
  }
  fill_tail_params(P, s, nu1, nu2, coarse_iters, symmetric, uo.data(), bo.data());
  return launch_coarse_tail<T>(P, stream);
}

template struct MGCore<float>;
template struct MGCore<double>;

// ------------------------------------------------------------------------------------------
// Driver (Sol_MultigridPressure3DBase)
// ------------------------------------------------------------------------------------------
CoreOps *MGSolver::active() {
  if (co) return co->ops();
  return double_mode ? (CoreOps *)&cd : (CoreOps *)&cf;
}

int MGSolver::coarse_iters() const {
  const int cl = num_levels - 1;
  int d[3];
  for (int q = 0; q < 3; q++) d[q] = co ? co->coarse_dim()[q] : (kind == OCU_MG_F32) ? cf.dim[cl][q] : cd.dim[cl][q];
  const int a = d[0] * d[1], b = d[1] * d[2], c = d[0] * d[2];
  const int mx = a > b ? (a > c ? a : c) : (b > c ? b : c);
  return mx / 2;
}

static double pick(int conv, double l2, double linf) {
  return (conv & OCU_CONVERGENCE_CRITERIA_L2) ? l2 : (conv & OCU_CONVERGENCE_CRITERIA_LINF) ? linf : 1e20;
}

// do_fmg (sol_mgpressure3d.cpp:113-251); returns OCU_OK (converged), OCU_ERR_NOT_CONVERGED, or
// an error.
// ------------------------------------------------------------------------------------------
// CUDA-graph replay.  The schedule between two host decisions is fixed for a given solver
// configuration, so each such segment is captured once (stream capture of the same enqueue
// code) and replayed with one cudaGraphLaunch:
//   INIT   ghost fill of u0 + residual norms of level 0 (read back, then decide)
//   RAMP   restriction chain + the FMG cycles from the coarsest level up to level 1
//   PRE0   pre-smooth at level 0, clear level 1, residual+restriction+norms (read back)
//   REST0  the rest of a level-0 cycle (levels 1.. down, tail kernel, up to level 0)
//   FINAL  ghost fill of u0 after convergence
// With CONVERGENCE_NONE nothing is read back, so a whole fixed-schedule FMG (the refinement
// solver's inner solve) runs as a chain of graph launches without a host wait.
// ------------------------------------------------------------------------------------------
MGSolver::~MGSolver() {
  co.reset();  // waits for every image's stream; image 0's pressure is freed below
  clear_graphs();
  if (stream) cudaStreamSynchronize(stream);
  if (pressure) { cudaFree(pressure->buf); delete pressure; }
  if (rhs_f) { cudaFree(rhs_f->buf); delete rhs_f; }
  if (own_stream) cudaStreamDestroy(own_stream);
}

void MGSolver::clear_graphs() {
  for (auto &kv : graphs) cudaGraphExecDestroy(kv.second.exec);
  graphs.clear();
}

template <typename F>
ocu_status MGSolver::run_segment(const void *core, int seg, F &&enqueue) {
  if (!use_graphs) return enqueue();
  const auto key = std::make_pair(core, seg);
  auto it = graphs.find(key);
  if (it == graphs.end()) {
    OCU_TRY(check_cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture"));
    set_capturing(true);
    const unsigned long long n0 = launch_count_captured();
    ocu_status st = co ? co->ops()->fork() : OCU_OK;
    if (st == OCU_OK) st = enqueue();
    if (st == OCU_OK && co) st = co->ops()->join();
    const int kernels = (int)(launch_count_captured() - n0);
    set_capturing(false);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (st != OCU_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    OCU_TRY(check_cuda(e, "cudaStreamEndCapture"));
    GraphEntry ent;
    e = cudaGraphInstantiate(&ent.exec, g, 0);
    cudaGraphDestroy(g);
    OCU_TRY(check_cuda(e, "cudaGraphInstantiate"));
    ent.kernels = kernels;
    it = graphs.emplace(key, ent).first;
  }
  OCU_TRY(check_cuda(cudaGraphLaunch(it->second.exec, stream), "cudaGraphLaunch"));
  count_launch(it->second.kernels);
  return OCU_OK;
}

enum { SEG_INIT = 0, SEG_RAMP = 8, SEG_PRE0 = 16, SEG_REST0 = 24, SEG_FINAL = 32 };

// levels [a, b) of a down-leg without norm checks
ocu_status MGSolver::enq_down(CoreOps *c, int a, int b) {
  for (int level = a; level < b; level++) {
    OCU_TRY(c->relax(level, prm.nu1, RO_RED_BLACK));
    OCU_TRY(c->clear_and_restrict(level, false, false));
  }
  return OCU_OK;
}

// tail from level s, then the up-leg from s-1 to f
ocu_status MGSolver::enq_tail_up(CoreOps *c, int s, int f) {
  const bool sym = prm.make_symmetric_operator != 0;
  OCU_TRY(c->cycle_tail(s, prm.nu1, prm.nu2, coarse_iters(), sym));
  for (int level = s - 1; level >= f; level--) {
    OCU_TRY(c->prolong(level + 1, level));
    if (level > 0) OCU_TRY(c->relax(level, prm.nu2, sym ? RO_BLACK_RED : RO_RED_BLACK));
  }
  return OCU_OK;
}

ocu_status MGSolver::do_fmg_graph(double tolerance, int max_iter, double *rl2, double *rlinf) {
  const int conv = prm.convergence;
  const bool wl2 = conv & OCU_CONVERGENCE_CALC_L2, wlinf = conv & OCU_CONVERGENCE_CALC_LINF;
  const int nv = (wl2 ? 1 : 0) + (wlinf ? 2 : 0);
  CoreOps *c = active();
  const int ts = c->tail_start();
  double orig_l2 = 0, orig_linf = 0;
  *rl2 = *rlinf = 0;
  OCU_TRY(run_segment(c, SEG_INIT + nv, [&]() -> ocu_status {
    OCU_TRY(c->apply_bc(0));
    return c->enqueue_restrict_residuals(0, 0, wl2, wlinf);
  }));
  if (wl2 || wlinf) OCU_TRY(c->finish_norms(0, wl2 ? &orig_l2 : nullptr, wlinf ? &orig_linf : nullptr));
  if (pick(conv, orig_l2, orig_linf) < tolerance) {
    if (wl2) *rl2 = orig_l2;
    if (wlinf) *rlinf = orig_linf;
    stats.vcycles = 0;
    return OCU_OK;
  }
  OCU_TRY(run_segment(c, SEG_RAMP, [&]() -> ocu_status {
    for (int level = 0; level < num_levels - 1; level++) {
      OCU_TRY(c->clear_and_restrict(level, false, false));
    }
    for (int f = num_levels - 1; f >= 1; f--) {
      const int s = ts > f ? ts : f;
      OCU_TRY(enq_down(c, f, s));
      OCU_TRY(enq_tail_up(c, s, f));
      OCU_TRY(c->prolong(f, f - 1));
    }
    return OCU_OK;
  }));
  int num_vcyc = 0;
  for (int i_cyc = 0; i_cyc < max_iter + 1; i_cyc++) {
    num_vcyc++;
    OCU_TRY(run_segment(c, SEG_PRE0 + nv, [&]() -> ocu_status {
      OCU_TRY(c->relax(0, prm.nu1, RO_RED_BLACK));
      return c->clear_and_restrict(0, wl2, wlinf);
    }));
    if (wl2 || wlinf) {
      OCU_TRY(c->finish_norms(0, wl2 ? rl2 : nullptr, wlinf ? rlinf : nullptr));
      stats.last_l2 = *rl2;
      stats.last_linf = *rlinf;
    }
    if (pick(conv, *rl2, *rlinf) < tolerance) {
      OCU_TRY(run_segment(c, SEG_FINAL, [&]() -> ocu_status { return c->apply_bc(0); }));
      stats.vcycles = num_vcyc;
      return OCU_OK;
    }
    OCU_TRY(run_segment(c, SEG_REST0, [&]() -> ocu_status {
      OCU_TRY(enq_down(c, 1, ts));
      return enq_tail_up(c, ts, 0);
    }));
  }
  stats.vcycles = num_vcyc;
  return OCU_ERR_NOT_CONVERGED;
}

ocu_status MGSolver::do_vcycle_graph(double tolerance, int max_iter, double *rl2, double *rlinf) {
  const int conv = prm.convergence;
  const bool wl2 = conv & OCU_CONVERGENCE_CALC_L2, wlinf = conv & OCU_CONVERGENCE_CALC_LINF;
  const int nv = (wl2 ? 1 : 0) + (wlinf ? 2 : 0);
  CoreOps *c = active();
  const int ts = c->tail_start();
  double orig_l2 = 0, orig_linf = 0;
  OCU_TRY(run_segment(c, SEG_INIT + nv, [&]() -> ocu_status {
    OCU_TRY(c->apply_bc(0));
    return c->enqueue_restrict_residuals(0, 0, wl2, wlinf);
  }));
  if (wl2 || wlinf) OCU_TRY(c->finish_norms(0, wl2 ? &orig_l2 : nullptr, wlinf ? &orig_linf : nullptr));
  if (pick(conv, orig_l2, orig_linf) < tolerance) {
    if (wl2) *rl2 = orig_l2;
    if (wlinf) *rlinf = orig_linf;
    return OCU_OK;
  }
  for (int i_cyc = 0; i_cyc < max_iter; i_cyc++) {
    OCU_TRY(run_segment(c, SEG_PRE0 + nv, [&]() -> ocu_status {
      OCU_TRY(c->relax(0, prm.nu1, RO_RED_BLACK));
      return c->clear_and_restrict(0, wl2, wlinf);
    }));
    if (wl2 || wlinf) OCU_TRY(c->finish_norms(0, wl2 ? rl2 : nullptr, wlinf ? rlinf : nullptr));
    if (pick(conv, *rl2, *rlinf) < tolerance) {
      OCU_TRY(run_segment(c, SEG_FINAL, [&]() -> ocu_status { return c->apply_bc(0); }));
      return OCU_OK;
    }
    OCU_TRY(run_segment(c, SEG_REST0, [&]() -> ocu_status {
      OCU_TRY(enq_down(c, 1, ts));
      return enq_tail_up(c, ts, 0);
    }));
  }
  return OCU_ERR_NOT_CONVERGED;
}

ocu_status MGSolver::do_fmg(double tolerance, int max_iter, double *rl2, double *rlinf) {
  if (use_graphs && num_levels >= 2) return do_fmg_graph(tolerance, max_iter, rl2, rlinf);
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
    OCU_TRY(c->clear_and_restrict(level, false, false));
  }
  for (int fine_level = num_levels - 1; fine_level >= 0; fine_level--) {
    const int level_ncyc = (fine_level == 0) ? max_iter + 1 : 1;
    for (int i_cyc = 0; i_cyc < level_ncyc; i_cyc++) {
      if (fine_level == 0) num_vcyc++;
      bool converged = false;
      OCU_TRY(cycle(c, fine_level, tolerance, rl2, rlinf, &converged));
      if (converged) {
        stats.vcycles = num_vcyc;
        return OCU_OK;
      }
    }
    if (fine_level > 0) OCU_TRY(c->prolong(fine_level, fine_level - 1));
  }
  stats.vcycles = num_vcyc;
  return OCU_ERR_NOT_CONVERGED;
}

// One V-cycle from fine_level (the body of the cycle loops of do_fmg and do_vcycle).  The
// levels from tail_start() down are handed to the single-CTA tail kernel; at level 0 the
// residual norm is read back after the pre-smooth and the cycle stops when it is below the
// tolerance, after refreshing the level-0 ghosts (sol_mgpressure3d.cpp:186-236).
ocu_status MGSolver::cycle(CoreOps *c, int fine_level, double tolerance, double *rl2, double *rlinf,
                           bool *converged) {
  const int conv = prm.convergence;
  const int coarse_level = num_levels - 1;
  const bool sym = prm.make_symmetric_operator != 0;
  const int s = c->tail_start() > fine_level ? c->tail_start() : fine_level;
  *converged = false;
  for (int level = fine_level; level < s; level++) {
    OCU_TRY(c->relax(level, prm.nu1, RO_RED_BLACK));
    if (level == 0) {
      double *l2 = (conv & OCU_CONVERGENCE_CALC_L2) ? rl2 : nullptr;
      double *linf = (conv & OCU_CONVERGENCE_CALC_LINF) ? rlinf : nullptr;
      OCU_TRY(c->clear_and_restrict(0, l2 != nullptr, linf != nullptr));
      if (l2 || linf) OCU_TRY(c->finish_norms(0, l2, linf));
      stats.last_l2 = *rl2;
      stats.last_linf = *rlinf;
      if (pick(conv, *rl2, *rlinf) < tolerance) {
        OCU_TRY(c->apply_bc(0));
        *converged = true;
        return OCU_OK;
      }
    } else {
      OCU_TRY(c->clear_and_restrict(level, false, false));
    }
  }
  OCU_TRY(c->cycle_tail(s, prm.nu1, prm.nu2, coarse_iters(), sym));
  (void)coarse_level;
  for (int level = s - 1; level >= fine_level; level--) {
    OCU_TRY(c->prolong(level + 1, level));
    if (level > 0) OCU_TRY(c->relax(level, prm.nu2, sym ? RO_BLACK_RED : RO_RED_BLACK));
  }
  return OCU_OK;
}

// do_vcycle (sol_mgpressure3d.cpp:253-329)
ocu_status MGSolver::do_vcycle(double tolerance, int max_iter, double *rl2, double *rlinf) {
  if (use_graphs && num_levels >= 2) return do_vcycle_graph(tolerance, max_iter, rl2, rlinf);
  const int conv = prm.convergence;
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
    bool converged = false;
    OCU_TRY(cycle(c, 0, tolerance, rl2, rlinf, &converged));
    if (converged) return OCU_OK;
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
  if (chq && prm.ir_inner_exact == 0) return ir_solve_chequer(tolerance, max_outer, rl2, rlinf);
  const int conv = prm.convergence;
  const ocu_layout &L = cd.lay[0];
  double l2 = 0, linf = 0;
  stats.outer_iterations = 0;
  stats.vcycles = 0;
  double_mode = true;
  OCU_TRY(cd.apply_bc(0));
  OCU_TRY(ir_residual(&l2, &linf));
  *rl2 = l2; *rlinf = linf;
  stats.last_l2 = l2; stats.last_linf = linf;
  if (pick(conv, l2, linf) < tolerance) return OCU_OK;
  const int inner = prm.ir_inner_cycles > 0 ? prm.ir_inner_cycles : 4;
  ocu_mg_params saved = prm;
  int total_inner = 0;
  (void)L;
  for (int outer = 1; outer <= max_outer; outer++) {
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
    OCU_TRY(ir_residual(&l2, &linf));
    stats.outer_iterations = outer;
    stats.vcycles = total_inner;
    *rl2 = l2; *rlinf = linf;
    stats.last_l2 = l2; stats.last_linf = linf;
    if (pick(conv, l2, linf) < tolerance) return OCU_OK;
  }
  return OCU_ERR_NOT_CONVERGED;
}

// The same refinement with the split-layout FP32 correction solver (ir_chequer.cu).  One
// captured graph per refinement step: FMG ramp + ir_inner_cycles fine-level V-cycles from a zero
// correction, x += e (fused into the last prolongation), the level-0 ghost refresh with the caller's boundary values, the FP64
// residual (written as float into the correction's right-hand side) and its norms.  The host
// waits once per step, for the norms.
enum { SEG_CHQ_FIRST = 0, SEG_CHQ_STEP = 1 };

ocu_status MGSolver::ir_chequer_residual_tail() {
  const ocu_layout &L = cd.lay[0];
  double *rows2 = (double *)cd.rows, *rowsinf = (double *)cd.rows + cd.rows_stride;
  const long long nrows = (long long)L.nx * L.ny;
  OCU_TRY(chq->enqueue_residual(cd.u0(0), cd.b0(0), L, cd.h[0], cd.fx, cd.fy, cd.fz, rows2, rowsinf, stream));
  OCU_TRY(launch_fold_rows<double>(rows2, nrows, false, cd.red_scratch, cd.d_norms, stream));
  OCU_TRY(launch_fold_rows<double>(rowsinf, nrows, true, cd.red_scratch, cd.d_norms + 1, stream));
  return launch_readback(cd.d_norms, cd.h_norms, 3, stream);
}

ocu_status MGSolver::ir_solve_chequer(double tolerance, int max_outer, double *rl2, double *rlinf) {
  const int conv = prm.convergence;
  double l2 = 0, linf = 0;
  stats.outer_iterations = 0;
  stats.vcycles = 0;
  double_mode = true;
  OCU_TRY(run_segment(chq.get(), SEG_CHQ_FIRST, [&]() -> ocu_status {
    OCU_TRY(cd.apply_bc(0));
    return ir_chequer_residual_tail();
  }));
  OCU_TRY(cd.finish_norms(0, &l2, &linf));
  *rl2 = l2; *rlinf = linf;
  stats.last_l2 = l2; stats.last_linf = linf;
  if (pick(conv, l2, linf) < tolerance) return OCU_OK;
  const int inner = prm.ir_inner_cycles > 0 ? prm.ir_inner_cycles : 4;
  const int citers = coarse_iters();
  for (int outer = 1; outer <= max_outer; outer++) {
    OCU_TRY(run_segment(chq.get(), SEG_CHQ_STEP, [&]() -> ocu_status {
      OCU_TRY(chq->enqueue_fmg(prm.nu1, prm.nu2, inner, citers, prm.nu1 + prm.nu2, stream, cd.u0(0), &cd.lay[0]));
      OCU_TRY(cd.apply_bc(0));
      return ir_chequer_residual_tail();
    }));
    OCU_TRY(cd.finish_norms(0, &l2, &linf));
    stats.outer_iterations = outer;
    stats.vcycles = outer * inner;
    *rl2 = l2; *rlinf = linf;
    stats.last_l2 = l2; stats.last_linf = linf;
    if (pick(conv, l2, linf) < tolerance) return OCU_OK;
  }
  return OCU_ERR_NOT_CONVERGED;
}

// FP64 residual of the refinement step, with both norms, written to the FP32 hierarchy's
// right-hand side as float in the same pass.
ocu_status MGSolver::ir_residual(double *l2, double *linf) {
  const ocu_layout &L = cd.lay[0];
  if (!cd.fused || cd.store_residuals) {
    OCU_TRY(cd.restrict_residuals(0, 0, l2, linf));
    return launch_downcast_interior((const double *)cd.r0(0), (float *)cf.b0(0), L, stream);
  }
  double *rows2 = (double *)cd.rows, *rowsinf = (double *)cd.rows + cd.rows_stride;
  OCU_TRY(launch_residual_rows<double>(cd.u0(0), cd.b0(0), nullptr, (float *)cf.b0(0), L, cd.h[0], cd.fx, cd.fy,
                                       cd.fz, rows2, rowsinf, stream));
  const long long nrows = (long long)L.nx * L.ny;
  OCU_TRY(launch_fold_rows<double>(rows2, nrows, false, cd.red_scratch, cd.d_norms, stream));
  OCU_TRY(launch_fold_rows<double>(rowsinf, nrows, true, cd.red_scratch, cd.d_norms + 1, stream));
  OCU_TRY(launch_readback(cd.d_norms, cd.h_norms, 3, stream));
  return cd.finish_norms(0, l2, linf);
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
  if (co && (st == OCU_OK || st == OCU_ERR_NOT_CONVERGED)) OCU_TRY(co->ops()->join());
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
  if (st == OCU_OK && co) st = co->ops()->join();
  if (st == OCU_OK) st = check_cuda(cudaStreamSynchronize(stream), "run_vcycles");
  return st;
}

ocu_status MGSolver::run_fmg(int count) {
  if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] run_fmg - not initialized");
  if (count < 0) return fail(OCU_ERR_INVALID_VALUE, "[WARNING] Sol_MultigridPressure3DDevice::run_fmg - negative count %d", count);
  double l2, linf;
  ocu_status st = do_fmg(0, count, &l2, &linf);
  if (st == OCU_ERR_NOT_CONVERGED) st = OCU_OK;
  if (st == OCU_OK && co) st = co->ops()->join();
  if (st == OCU_OK) st = check_cuda(cudaStreamSynchronize(stream), "run_fmg");
  return st;
}

ocu_status MGSolver::initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, ocu_grid *rhs) {
  if (initialized) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] initialize_storage - already initialized");
  if (co_images > 0)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] initialize_storage - a multi-image solver takes one rhs per image (ocu_mgco_initialize_storage)");
  if (!stream) set_stream(nullptr);
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
      cf.d_err = cd.d_err;  // one timeout word, read back with the FP64 norms
      if (kind == OCU_MG_MIXED_IR && ChequerMG::suits(cd.dim, fbc)) {
        chq.reset(new ChequerMG());
        OCU_TRY(chq->init(cd.dim, cd.h, cd.fx, cd.fy, cd.fz, cd.omega, fbc));
      }
    }
  }
  stats.num_levels = num_levels;
  OCU_TRY(apply_knobs());
  initialized = true;
  return OCU_OK;
}

ocu_status MGSolver::apply_knobs() {
  const int tc = prm.tail_cells == 0 ? kDefaultTailCells : (prm.tail_cells < 0 ? 0 : prm.tail_cells);
  cf.fused = cd.fused = prm.unfused == 0;
  cf.store_residuals = cd.store_residuals = prm.store_residual_grids != 0;
  cf.tail_cells = cd.tail_cells = tc;
  cf.sweep_cells = cd.sweep_cells = prm.sweep_cells <= 0 ? kDefaultSweepCells : prm.sweep_cells;
  if (cf.sweep_cells > 0 && cf.num_levels > 0) OCU_TRY(cf.ensure_sweep_buffers());
  if (cd.sweep_cells > 0 && cd.num_levels > 0) OCU_TRY(cd.ensure_sweep_buffers());
  cf.wait_limit = cd.wait_limit = prm.wait_limit;
  return OCU_OK;
}

ocu_status MGSolver::set_params(const ocu_mg_params &p) {
  // unchanged parameters keep the recorded graphs (callers may re-send them before every solve)
  if (initialized && std::memcmp(&p, &prm, sizeof(p)) == 0) return OCU_OK;
  prm = p;
  cf.bc = p.bc;
  cd.bc = p.bc;
  if (kind == OCU_MG_MIXED_IR) bc_make_homogeneous(&cf.bc);
  cf.disable_relax_on_host = cd.disable_relax_on_host = p.disable_relax_on_host != 0;
  if (co) co->ops()->on_params(p);
  clear_graphs();  // captured schedules depend on every parameter
  return apply_knobs();
}

// Work runs on the caller's stream.  The legacy default stream (NULL) cannot be captured into a
// graph, so for NULL the solver uses a private blocking stream, which the legacy stream orders
// against implicitly in both directions -- the same semantics as issuing on NULL.
void MGSolver::set_stream(cudaStream_t s) {
  if (!s) {
    if (!own_stream) cudaStreamCreate(&own_stream);
    s = own_stream;
  }
  stream = s;
  cf.stream = s;
  cd.stream = s;
  if (co) co->ops()->on_stream(s);
}

// Sol_MultigridPressure3DDeviceCo::initialize_storage (sol_mgpressure3dco.cu:240-520)
ocu_status MGSolver::initialize_storage_co(int nxl, int ny, int nz, double hx, double hy, double hz,
                                           ocu_grid *const *rhs) {
  if (initialized) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] initialize_storage - already initialized");
  if (!rhs) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDeviceCo::initialize_storage - null rhs");
  const ocu_dtype want = kind == OCU_MG_F32 ? OCU_F32 : OCU_F64;
  for (int i = 0; i < co_images; i++) {
    const ocu_grid *r = rhs[i];
    if (!r) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDeviceCo::initialize_storage - null rhs of image %d", i);
    if (r->dtype != want) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDeviceCo::initialize_storage - rhs dtype mismatch (image %d)", i);
    if (r->L.gx < 1 || r->L.gy < 1 || r->L.gz < 1)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDevice::initialize_storage - rhs has invalid ghost cells (%d,%d,%d), must be >= 1", r->L.gx, r->L.gy, r->L.gz);
    if (r->L.nx != nxl || r->L.ny != ny || r->L.nz != nz)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDevice::initialize_storage - rhs dimension mismatch (%d,%d,%d) != (%d,%d,%d)", r->L.nx, r->L.ny, r->L.nz, nxl, ny, nz);
    const ocu_layout &a = r->L, &b = rhs[0]->L;
    if (a.gx != b.gx || a.gy != b.gy || a.gz != b.gz || a.pnx != b.pnx || a.pny != b.pny || a.pnz != b.pnz)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDeviceCo::initialize_storage - the images' rhs layouts differ (image %d)", i);
  }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(co_devices[0]);
  if (!stream) set_stream(nullptr);
  ocu_status st = OCU_OK;
  pressure = alloc_grid(want, rhs[0]->L, &st);
  if (pressure) st = mgco_create(want, co_images, co_devices.data(), nxl, ny, nz, hx, hy, hz, rhs, pressure, prm,
                                 co_cutoff_cells, stream, &co);
  cudaSetDevice(prev);
  if (st != OCU_OK) {
    co.reset();
    return st;
  }
  num_levels = co->ops()->levels();
  double_mode = kind != OCU_MG_F32;
  // segments are captured across the images' streams (fork / join) when the images share one
  // device; images on several devices run without replay
  for (int d : co_devices)
    if (d != co_devices[0]) use_graphs = false;
  stats.num_levels = num_levels;
  {
    const double h0 = hx < hy ? (hx < hz ? hx : hz) : (hy < hz ? hy : hz);
    stats.omega = mg_optimal_omega(h0 * h0 / (hx * hx), h0 * h0 / (hy * hy), h0 * h0 / (hz * hz));
  }
  initialized = true;
  return OCU_OK;
}

ocu_grid *MGSolver::level_grid(char which, int level) {
  if (!initialized || level < 0 || level >= num_levels) return nullptr;
  if (co) return co->ops()->grid(which, level);
  auto &core = (kind == OCU_MG_F32) ? (CoreOps &)cf : (CoreOps &)cd;
  return core.grid(which, level);
}

}  // namespace ocub
