// Projection (Sol_ProjectDivergence3DDevice<T>) and the Boussinesq Navier-Stokes stepper
// (Eqn_IncompressibleNS3D<T>) over the sm_100a stencil kernels and the multigrid solver.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "flow_solvers.h"

namespace ocub {

static bool valid_mac(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w, int nx, int ny, int nz) {
  // check_valid_mac_dimensions (ocustorage/grid3dops.cpp:24-45)
  if (u->L.nx != nx + 1 || u->L.ny != ny || u->L.nz != nz) return false;
  if (v->L.nx != nx || v->L.ny != ny + 1 || v->L.nz != nz) return false;
  if (w->L.nx != nx || w->L.ny != ny || w->L.nz != nz + 1) return false;
  return layout_match(u->L, v->L) && layout_match(u->L, w->L);
}

// convert_bc_to_poisson_eqn (sol_project3d.cpp:26-43)
static bool convert_bc(const ocu_bc &b, ocu_bc *out) {
  out->type = OCU_BC_INVALID;
  out->value = 0;
  out->aux_value = 0;
  if (b.type == OCU_BC_PERIODIC) { out->type = OCU_BC_PERIODIC; return true; }
  if (b.type == OCU_BC_FORCED_INFLOW_VARIABLE_SLIP) { out->type = OCU_BC_NEUMANN; return true; }
  return false;
}

ProjectSolver::~ProjectSolver() {
  delete mg;
  if (divergence) { cudaFree(divergence->buf); delete divergence; }
  if (divergence64) { cudaFree(divergence64->buf); delete divergence64; }
}

// initialize_storage (sol_project3ddev.cu:100-135, initialize_device_storage :28-53; the mixed
// class, sol_projectmixed3d.cu:48-91, differs only in its pressure solver)
ocu_status ProjectSolver::initialize_storage(int nx_, int ny_, int nz_, double hx_, double hy_, double hz_,
                                             ocu_grid *u_, ocu_grid *v_, ocu_grid *w_, const ocu_bc_set &bc_) {
  if (!u_ || !v_ || !w_) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_ProjectDivergence3DDevice::initialize_storage - null grid");
  if (u_->dtype != dtype || v_->dtype != dtype || w_->dtype != dtype)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_ProjectDivergence3DDevice::initialize_storage - element type mismatch");
  if (!valid_mac(u_, v_, w_, nx_, ny_, nz_))
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_ProjectDivergence3DBase::initialize_base_storage - u,v,w grid dimensions mismatch");
  if (!check_float((float)hx_) || !check_float((float)hy_) || !check_float((float)hz_))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_ProjectDivergence3DBase::initialize_base_storage - garbage hx,hy,hz value");
  if (u_->L.gx < 1 || u_->L.gy < 1 || u_->L.gz < 1)
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_Divergence3DDevice::initialize_storage - must have at least one ghost cell on all sides");
  nx = nx_; ny = ny_; nz = nz_;
  hx = hx_; hy = hy_; hz = hz_;
  u = u_; v = v_; w = w_;
  bc = bc_;
  ocu_mg_params p;
  ocu_mg_params_default(&p);
  if (!convert_bc(bc.xneg, &p.bc.xneg) || !convert_bc(bc.xpos, &p.bc.xpos) || !convert_bc(bc.yneg, &p.bc.yneg) ||
      !convert_bc(bc.ypos, &p.bc.ypos) || !convert_bc(bc.zneg, &p.bc.zneg) || !convert_bc(bc.zpos, &p.bc.zpos))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_ProjectDivergence3DBase::convert_bc_to_poisson_eqn - invalid boundary condition type");
  ocu_layout Ld;
  layout_compute(nx, ny, nz, 1, 1, 1, u->L.pnx - (nx + 2), u->L.pny - (ny + 2), u->L.pnz - (nz + 2), &Ld);
  if (!layout_match(Ld, u->L))
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_ProjectDivergence3DDevice::initialize_device_storage - divergence layout mismatch");
  divergence = new ocu_grid{dtype, Ld, nullptr, true};
  OCU_TRY(check_cuda(cudaMalloc(&divergence->buf, dtype_size(dtype) * Ld.allocated), "cudaMalloc(divergence)"));
  OCU_TRY(check_cuda(cudaMemset(divergence->buf, 0, dtype_size(dtype) * Ld.allocated), "cudaMemset(divergence)"));
  mg = new ocu_mg(mg_kind >= 0 ? (ocu_mg_kind)mg_kind : (dtype == OCU_F64 ? OCU_MG_F64 : OCU_MG_F32), p);
  mg->s.set_stream(stream);
  ocu_grid *rhs = divergence;
  if (p64()) {  // FP32 fields, FP64 pressure: the pressure solve reads an FP64 copy of the divergence
    divergence64 = new ocu_grid{OCU_F64, Ld, nullptr, true};
    OCU_TRY(check_cuda(cudaMalloc(&divergence64->buf, 8 * Ld.allocated), "cudaMalloc(divergence64)"));
    OCU_TRY(check_cuda(cudaMemset(divergence64->buf, 0, 8 * Ld.allocated), "cudaMemset(divergence64)"));
    rhs = divergence64;
  }
  OCU_TRY(mg->s.initialize_storage(nx, ny, nz, hx, hy, hz, rhs));
  if (!layout_match(u->L, mg->s.pressure->L))
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_ProjectDivergence3DDevice::initialize_storage - pressure layout mismatch");
  // pressure().clear_zero(); convergence = CONVERGENCE_LINF (sol_project3ddev.cu:131-132)
  OCU_TRY(check_cuda(cudaMemsetAsync(mg->s.pressure->buf, 0, dtype_size(mg->s.pressure->dtype) * Ld.allocated, stream),
                     "clear_zero"));
  p.convergence = OCU_CONVERGENCE_LINF;
  mg->s.set_params(p);
  initialized = true;
  return OCU_OK;
}

template <typename T>
ocu_status ProjectSolver::divergence_only_t() {
  OCU_TRY(launch_mac_bc_level1<T>(origin<T>(u), origin<T>(v), origin<T>(w), u->L, nx, ny, nz, bc, stream));
  return launch_divergence<T>(origin<T>(u), origin<T>(v), origin<T>(w), origin<T>(divergence), u->L, nx, ny, nz, hx,
                              hy, hz, stream);
}

template <typename T>
ocu_status ProjectSolver::solve_t(double tolerance) {
  OCU_TRY(divergence_only_t<T>());
  double residual = 0;
  ocu_status st = mg->s.solve(&residual, tolerance, 15);
  if (st != OCU_OK && st != OCU_ERR_NOT_CONVERGED) return st;
  OCU_TRY(launch_gradient<T>(origin<T>(u), origin<T>(v), origin<T>(w), origin<T>(mg->s.pressure), u->L, nx, ny, nz,
                             hx, hy, hz, (T)-1, stream));
  OCU_TRY(launch_mac_bc_level1<T>(origin<T>(u), origin<T>(v), origin<T>(w), u->L, nx, ny, nz, bc, stream));
  return st;
}

// solve (sol_project3ddev.cu:58-71): MAC ghosts, divergence, pressure solve (max_iter 15),
// u -= grad p, MAC ghosts.  A pressure solve that stops above tolerance makes the whole call
// report OCU_ERR_NOT_CONVERGED, as the reference returns false.
ocu_status ProjectSolver::solve(double tolerance) {
  if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] Sol_ProjectDivergence3DDevice::solve - not initialized");
  if (p64()) return solve_f32_p64(tolerance);
  return dtype == OCU_F64 ? solve_t<double>(tolerance) : solve_t<float>(tolerance);
}

// FP32 fields with the pressure solved by FP32 V-cycles inside FP64 refinement (a library
// option, no reference counterpart): the same steps as solve_t<float>, with the FP32
// divergence widened to double for the pressure solve and the FP64 pressure gradient applied to
// the FP32 velocity in double.
ocu_status ProjectSolver::solve_f32_p64(double tolerance) {
  OCU_TRY(divergence_only_t<float>());
  OCU_TRY(launch_convert<double, float>((double *)divergence64->buf, (const float *)divergence->buf,
                                        divergence->L.allocated, stream));
  double residual = 0;
  ocu_status st = mg->s.solve(&residual, tolerance, 15);
  if (st != OCU_OK && st != OCU_ERR_NOT_CONVERGED) return st;
  OCU_TRY(launch_gradient_p64(origin<float>(u), origin<float>(v), origin<float>(w), origin<double>(mg->s.pressure),
                              u->L, nx, ny, nz, hx, hy, hz, -1.0, stream));
  OCU_TRY(launch_mac_bc_level1<float>(origin<float>(u), origin<float>(v), origin<float>(w), u->L, nx, ny, nz, bc, stream));
  return st;
}

ocu_status ProjectSolver::solve_divergence_only() {
  if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] solve_divergence_only - not initialized");
  OCU_TRY(dtype == OCU_F64 ? divergence_only_t<double>() : divergence_only_t<float>());
  return check_cuda(cudaStreamSynchronize(stream), "solve_divergence_only");
}

void ProjectSolver::set_stream(cudaStream_t s) {
  stream = s;
  if (mg) mg->s.set_stream(s);
}

// ------------------------------------------------------------------------------------------
// Eqn_IncompressibleNS3D<T>
// ------------------------------------------------------------------------------------------
static double round_t(ocu_dtype dt, double x) { return dt == OCU_F64 ? x : (double)(float)x; }

NSSolver::~NSSolver() {
  drop_tail_graphs();
  for (ocu_grid *g : {u, v, w, t, du, dv, dw, dt, ldu, ldv, ldw, ldt}) {
    if (g) { cudaFree(g->buf); delete g; }
  }
  if (scratch) cudaFree(scratch);
  if (d_red) cudaFree(d_red);
  if (h_red) cudaFreeHost(h_red);
  if (d_coef) cudaFree(d_coef);
}

void NSSolver::drop_tail_graphs() {
  for (int q = 0; q < 4; q++) {
    if (tail_exec[q]) cudaGraphExecDestroy(tail_exec[q]);
    tail_exec[q] = nullptr;
    tail_seen[q] = 0;
  }
}

static ocu_status make_grid(ocu_dtype dt, const ocu_layout &L, ocu_grid **out) {
  ocu_grid *g = new ocu_grid{dt, L, nullptr, true};
  cudaError_t e = cudaMalloc(&g->buf, dtype_size(dt) * L.allocated);
  if (e != cudaSuccess) { delete g; return check_cuda(e, "cudaMalloc"); }
  e = cudaMemset(g->buf, 0, dtype_size(dt) * L.allocated);
  *out = g;
  return check_cuda(e, "cudaMemset");
}

ocu_status ns_init_layout(int nx, int ny, int nz, char which, ocu_layout *L) {
  // Eqn_IncompressibleNS3DParams::init_grids (eqn_incompressns3d.h:75-83)
  switch (which) {
    case 'u': layout_compute(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1, L); return OCU_OK;
    case 'v': layout_compute(nx, ny + 1, nz, 1, 1, 1, 1, 0, 1, L); return OCU_OK;
    case 'w': layout_compute(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0, L); return OCU_OK;
    case 't': layout_compute(nx, ny, nz, 1, 1, 1, 1, 1, 1, L); return OCU_OK;
    default: return fail(OCU_ERR_INVALID_VALUE, "[ERROR] init_grids - unknown grid '%c'", which);
  }
}

// set_parameters (eqn_incompressns3d.cu:164-298, set_base_parameters :67-117)
ocu_status NSSolver::set_parameters(const ocu_ns_params &p, const void *iu, const void *iv, const void *iw,
                                    const void *it) {
  if (!check_float((float)p.max_divergence) || p.max_divergence < 0 || p.max_divergence > 1)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - invalid max_divergence %f", p.max_divergence);
  if (p.cfl_factor < 0)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - invalid cfl_factor %f", p.cfl_factor);
  if (p.time_step != OCU_TS_ADAMS_BASHFORD2 && p.time_step != OCU_TS_FORWARD_EULER)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - unknown timestep type %d", p.time_step);
  const int vd = p.vertical_direction;
  if (vd != OCU_DIR_XPOS && vd != OCU_DIR_XNEG && vd != OCU_DIR_YPOS && vd != OCU_DIR_YNEG && vd != OCU_DIR_ZPOS &&
      vd != OCU_DIR_ZNEG)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - bad vertical_direction %d", vd);
  if (!check_float((float)p.hx) || !check_float((float)p.hy) || !check_float((float)p.hz) || p.hx <= 0 || p.hy <= 0 ||
      p.hz <= 0)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - bad hx, hy, hz (%f, %f, %f)", p.hx, p.hy, p.hz);
  if (!check_float((float)p.thermal_diffusion) || p.thermal_diffusion < 0)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - invalid thermal diffusion %f", p.thermal_diffusion);
  if (!check_float((float)p.viscosity) || p.viscosity < 0)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - invalid viscosity %f", p.viscosity);
  if (p.advection_scheme != OCU_IT_FIRST_ORDER_UPWIND && p.advection_scheme != OCU_IT_SECOND_ORDER_CENTERED)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - invalid interpolation type %d", p.advection_scheme);
  if (!bc_check_scalar(p.temp_bc) || !bc_check_mac(p.flow_bc))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Eqn_IncompressibleNS3D::set_parameters - invalid boundary condition types");
  if (!stream) set_stream(nullptr);
  prm = p;
  T_gravity = round_t(dtype, p.gravity);
  T_bouyancy = round_t(dtype, p.bouyancy);
  T_kappa = round_t(dtype, p.thermal_diffusion);
  T_nu = round_t(dtype, p.viscosity);
  lastdt = 0;
  num_steps = 0;
  swaps = 0;
  drop_tail_graphs();
  ocu_layout Lu, Lv, Lw, Lt;
  ns_init_layout(p.nx, p.ny, p.nz, 'u', &Lu);
  ns_init_layout(p.nx, p.ny, p.nz, 'v', &Lv);
  ns_init_layout(p.nx, p.ny, p.nz, 'w', &Lw);
  ns_init_layout(p.nx, p.ny, p.nz, 't', &Lt);
  OCU_TRY(make_grid(dtype, Lu, &u)); OCU_TRY(make_grid(dtype, Lu, &du)); OCU_TRY(make_grid(dtype, Lu, &ldu));
  OCU_TRY(make_grid(dtype, Lv, &v)); OCU_TRY(make_grid(dtype, Lv, &dv)); OCU_TRY(make_grid(dtype, Lv, &ldv));
  OCU_TRY(make_grid(dtype, Lw, &w)); OCU_TRY(make_grid(dtype, Lw, &dw)); OCU_TRY(make_grid(dtype, Lw, &ldw));
  OCU_TRY(make_grid(dtype, Lt, &t)); OCU_TRY(make_grid(dtype, Lt, &dt)); OCU_TRY(make_grid(dtype, Lt, &ldt));
  const size_t es = dtype_size(dtype);
  OCU_TRY(check_cuda(cudaMemcpy(u->buf, iu, es * Lu.allocated, cudaMemcpyHostToDevice), "copy init_u"));
  OCU_TRY(check_cuda(cudaMemcpy(v->buf, iv, es * Lv.allocated, cudaMemcpyHostToDevice), "copy init_v"));
  OCU_TRY(check_cuda(cudaMemcpy(w->buf, iw, es * Lw.allocated, cudaMemcpyHostToDevice), "copy init_w"));
  OCU_TRY(check_cuda(cudaMemcpy(t->buf, it, es * Lt.allocated, cudaMemcpyHostToDevice), "copy init_temp"));
  proj.dtype = dtype;
  proj.mg_kind = p.mixed_pressure ? OCU_MG_MIXED_IR : -1;
  proj.set_stream(stream);
  OCU_TRY(proj.initialize_storage(p.nx, p.ny, p.nz, p.hx, p.hy, p.hz, u, v, w, p.flow_bc));
  if (dtype == OCU_F64) {
    OCU_TRY(launch_mac_bc_level1<double>(origin<double>(u), origin<double>(v), origin<double>(w), Lu, p.nx, p.ny, p.nz, p.flow_bc, stream));
    OCU_TRY(launch_bc_level1<double>(origin<double>(t), Lt, p.temp_bc, p.hx, p.hy, p.hz, stream));
  } else {
    OCU_TRY(launch_mac_bc_level1<float>(origin<float>(u), origin<float>(v), origin<float>(w), Lu, p.nx, p.ny, p.nz, p.flow_bc, stream));
    OCU_TRY(launch_bc_level1<float>(origin<float>(t), Lt, p.temp_bc, p.hx, p.hy, p.hz, stream));
  }
  for (ocu_grid *g : {du, dv, dw, dt})
    OCU_TRY(check_cuda(cudaMemsetAsync(g->buf, 0, es * g->L.allocated, stream), "clear derivatives"));
  if (!scratch) {
    OCU_TRY(check_cuda(cudaMalloc(&scratch, reduce_scratch_bytes(Lu, 8) * 3), "cudaMalloc(ns scratch)"));
    OCU_TRY(check_cuda(cudaMemset(scratch, 0, reduce_scratch_bytes(Lu, 8) * 3), "cudaMemset"));
    OCU_TRY(check_cuda(cudaMalloc(&d_red, 4 * sizeof(double)), "cudaMalloc"));
    OCU_TRY(check_cuda(cudaMemset(d_red, 0, 4 * sizeof(double)), "cudaMemset"));
    OCU_TRY(check_cuda(cudaMallocHost(&h_red, 4 * sizeof(double)), "cudaMallocHost"));
    OCU_TRY(check_cuda(cudaMalloc(&d_coef, 4 * sizeof(double)), "cudaMalloc(step coefficients)"));
  }
  initialized = true;
  return check_cuda(cudaStreamSynchronize(stream), "set_parameters");
}

// get_max_stable_timestep (eqn_incompressns3d.cu:301-328)
ocu_status NSSolver::get_max_stable_timestep(double *out) {
  if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] get_max_stable_timestep - not initialized");
  // max |u|, max |v|, max |w| in one launch (the reference's three reduce_maxabs calls; a maximum
  // is the same in any fold order)
  const ocu_layout *lays[3] = {&u->L, &v->L, &w->L};
  if (dtype == OCU_F64) {
    const double *o[3] = {origin<double>(u), origin<double>(v), origin<double>(w)};
    OCU_TRY(launch_minmax<double>(o, lays, 3, OCU_REDUCE_MAXABS, scratch, d_red, stream));
  } else {
    const float *o[3] = {origin<float>(u), origin<float>(v), origin<float>(w)};
    OCU_TRY(launch_minmax<float>(o, lays, 3, OCU_REDUCE_MAXABS, scratch, d_red, stream));
  }
  // d_red[3] holds the timeout word of the TMA-fed advection (read with the maxima)
  OCU_TRY(launch_readback(d_red, h_red, 4, stream));
  OCU_TRY(check_cuda(cudaStreamSynchronize(stream), "maxabs"));
  if (*reinterpret_cast<const int *>(h_red + 3) != 0) {
    OCU_TRY(check_cuda(cudaMemsetAsync(d_red + 3, 0, sizeof(double), stream), "clear timeout word"));
    *reinterpret_cast<int *>(h_red + 3) = 0;
    return fail(OCU_ERR_TIMEOUT, "[ERROR] Eqn_IncompressibleNS3D - a load wait of the TMA-fed advection gave up (previous step)");
  }
  double ut = prm.hx / h_red[0], vt = prm.hy / h_red[1], wt = prm.hz / h_red[2];
  if (!check_float((float)ut)) ut = 1e10;
  if (!check_float((float)vt)) vt = 1e10;
  if (!check_float((float)wt)) wt = 1e10;
  auto min3 = [](double a, double b, double c) { return a < b ? (a < c ? a : c) : (b < c ? b : c); };
  double step = prm.cfl_factor * min3(ut, vt, wt);
  const double minh = min3(prm.hx, prm.hy, prm.hz);
  if (T_kappa > 0) step = std::min(step, (minh * minh) / round_t(dtype, 6 * T_kappa));
  if (T_nu > 0) step = std::min(step, (minh * minh) / round_t(dtype, 6 * T_nu));
  *out = step;
  return OCU_OK;
}

template <typename T>
ocu_status NSSolver::enqueue_tail(double dtv, T ab, bool ab2, const T *dcoef) {
  const int nx = prm.nx, ny = prm.ny, nz = prm.nz;
  const int vd = prm.vertical_direction;
  const ocu_layout &Lu = u->L;
  const T dm = (vd & OCU_DIR_NEGATIVE_FLAG) ? (T)1 : (T)-1;
  const T coef = dm * (T)T_gravity * (T)T_bouyancy;
  ocu_grid *vert = (vd & OCU_DIR_XAXIS_FLAG) ? du : (vd & OCU_DIR_YAXIS_FLAG) ? dv : dw;
  const int nbr = (vd & OCU_DIR_XAXIS_FLAG) ? t->L.xstride : (vd & OCU_DIR_YAXIS_FLAG) ? t->L.ystride : 1;
  // the step's coefficients: values, or slots 0, 1, 2 of dcoef (read when the kernels run)
  const Coef<T> c_dt = dcoef ? Coef<T>((T)dtv, dcoef + 0) : Coef<T>((T)dtv);
  const Coef<T> c_dab = dcoef ? Coef<T>((T)(dtv - ab), dcoef + 1) : Coef<T>((T)(dtv - ab));
  const Coef<T> c_ab = dcoef ? Coef<T>(ab, dcoef + 2) : Coef<T>(ab);
  // FP32 on a large grid: the TMA-fed form (bit-identical), its timeout word in d_red[3]
  ocu_status adv = OCU_ERR_UNSUPPORTED;
  if constexpr (sizeof(T) == 4) {
    const char *st = std::getenv("OCU_B200_TMA_STALL_TEST");  // polls; testing the timeout path
    adv = launch_advect_self_tma(origin<float>(u), origin<float>(v), origin<float>(w), origin<float>(du),
                                 origin<float>(dv), origin<float>(dw), Lu, nx, ny, nz, prm.hx, prm.hy, prm.hz,
                                 prm.advection_scheme, reinterpret_cast<int *>(d_red + 3), st ? -std::atoi(st) : 0,
                                 stream);
    if (adv != OCU_OK && adv != OCU_ERR_UNSUPPORTED) return adv;
  }
  if (adv == OCU_ERR_UNSUPPORTED)
    OCU_TRY(launch_advect_self<T>(origin<T>(u), origin<T>(v), origin<T>(w), origin<T>(du), origin<T>(dv),
                                  origin<T>(dw), Lu, nx, ny, nz, prm.hx, prm.hy, prm.hz, prm.advection_scheme, stream));
  // viscosity, then buoyancy on the vertical component; in FP32 the vertical component's two
  // passes are one kernel (same arithmetic, in the same order)
  bool buoyancy_done = false;
  if (T_nu > 0) {
    ocu_grid *st3[3] = {u, v, w}, *ds3[3] = {du, dv, dw};
    for (int c = 0; c < 3; c++) {
      const int ex = nx + (c == 0), ey = ny + (c == 1), ez = nz + (c == 2);
      if constexpr (sizeof(T) == 4) {
        if (ds3[c] == vert) {
          const ocu_status fs = launch_laplacian_thermal(origin<float>(st3[c]), origin<float>(ds3[c]), Lu, ex, ey, ez,
                                                         prm.hx, prm.hy, prm.hz, (float)T_nu, origin<float>(t),
                                                         (float)coef, nbr, nx, ny, nz, stream);
          if (fs == OCU_OK) {
            buoyancy_done = true;
            continue;
          }
          if (fs != OCU_ERR_UNSUPPORTED) return fs;
        }
      }
      OCU_TRY(launch_laplacian<T>(origin<T>(st3[c]), origin<T>(ds3[c]), Lu, ex, ey, ez, prm.hx, prm.hy, prm.hz,
                                  (T)T_nu, stream));
    }
  }
  if (!buoyancy_done)
    OCU_TRY(launch_thermal_force<T>(origin<T>(vert), coef, origin<T>(t), t->L, nbr, nx, ny, nz, stream));
  OCU_TRY(launch_advect_passive<T>(origin<T>(u), origin<T>(v), origin<T>(w), origin<T>(t), origin<T>(dt), t->L, nx, ny,
                                   nz, prm.hx, prm.hy, prm.hz, prm.advection_scheme, stream));
  if (T_kappa > 0)
    OCU_TRY(launch_laplacian<T>(origin<T>(t), origin<T>(dt), t->L, nx, ny, nz, prm.hx, prm.hy, prm.hz, (T)T_kappa, stream));
  T *tb = (T *)t->buf;
  if (ab2) {
    OCU_TRY(launch_lincomb2<T>(tb, t->L, (T)1.0, tb, c_dab, (const T *)dt->buf, stream));
    OCU_TRY(launch_lincomb2<T>(tb, t->L, (T)1.0, tb, c_ab, (const T *)ldt->buf, stream));
  } else {
    OCU_TRY(launch_lincomb2<T>(tb, t->L, (T)1.0, tb, c_dt, (const T *)dt->buf, stream));
  }
  OCU_TRY(launch_bc_nocorners_dev<T>(origin<T>(t), t->L, prm.temp_bc, prm.hx, prm.hy, prm.hz, stream));
  ocu_grid *st[3] = {u, v, w}, *ds[3] = {du, dv, dw}, *ls[3] = {ldu, ldv, ldw};
  // u, v, w updated in one pass when they take the interior 16-byte form
  {
    T *x3[3] = {(T *)u->buf, (T *)v->buf, (T *)w->buf};
    const T *d3[3] = {(const T *)du->buf, (const T *)dv->buf, (const T *)dw->buf};
    const T *l3[3] = {(const T *)ldu->buf, (const T *)ldv->buf, (const T *)ldw->buf};
    const ocu_status us = ab2 ? launch_update3<T>(x3, d3, l3, Lu, c_dab, c_ab, stream)
                              : launch_update3<T>(x3, d3, nullptr, Lu, c_dt, Coef<T>((T)0), stream);
    if (us == OCU_OK) return OCU_OK;
    if (us != OCU_ERR_UNSUPPORTED) return us;
  }
  for (int c = 0; c < 3; c++) {
    T *x = (T *)st[c]->buf;
    if (ab2) {
      OCU_TRY(launch_lincomb2<T>(x, st[c]->L, (T)1.0, x, c_dab, (const T *)ds[c]->buf, stream));
      OCU_TRY(launch_lincomb2<T>(x, st[c]->L, (T)1.0, x, c_ab, (const T *)ls[c]->buf, stream));
    } else {
      OCU_TRY(launch_lincomb2<T>(x, st[c]->L, (T)1.0, x, c_dt, (const T *)ds[c]->buf, stream));
    }
  }
  return OCU_OK;
}

static __global__ void k_set_coef(double *c, double a, double b, double d) {
  c[0] = a; c[1] = b; c[2] = d;
}
static __global__ void k_set_coef(float *c, float a, float b, float d) {
  c[0] = a; c[1] = b; c[2] = d;
}

// Environment read by the tail's launchers (the TMA advection's mode and its timeout test): a
// graph captured under one setting is not replayed under another.
static std::string tail_env_signature() {
  std::string sig;
  for (const char *k : {"OCU_B200_ADVECT_TMA", "OCU_B200_TMA_STALL_TEST"}) {
    const char *v = std::getenv(k);
    sig += v ? v : "-";
    sig += ';';
  }
  return sig;
}

// The step's coefficients into d_coef, then the state's graph (captured on first use).
template <typename T>
ocu_status NSSolver::replay_tail(int key, double dtv, T ab, bool ab2) {
  T *c = reinterpret_cast<T *>(d_coef);
  k_set_coef<<<1, 1, 0, stream>>>(c, (T)dtv, (T)(dtv - ab), ab);
  OCU_TRY(check_launch("k_set_coef"));
  if (!tail_exec[key]) {
    OCU_TRY(check_cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture"));
    set_capturing(true);
    const unsigned long long n0 = launch_count_captured();
    const ocu_status st = enqueue_tail<T>(dtv, ab, ab2, c);
    tail_kernels[key] = (int)(launch_count_captured() - n0);
    set_capturing(false);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (st != OCU_OK || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return st != OCU_OK ? st : check_cuda(e, "cudaStreamEndCapture");
    }
    e = cudaGraphInstantiate(&tail_exec[key], g, 0);
    cudaGraphDestroy(g);
    OCU_TRY(check_cuda(e, "cudaGraphInstantiate"));
  }
  OCU_TRY(check_cuda(cudaGraphLaunch(tail_exec[key], stream), "cudaGraphLaunch"));
  count_launch(tail_kernels[key]);
  return OCU_OK;
}

// advance_one_step (eqn_incompressns3d.cu:331-399): the tail (advection, diffusion, buoyancy,
// updates, temperature ghosts) as plain launches or one graph replay, then the projection.
template <typename T>
ocu_status NSSolver::step_t(double dtv) {
  const T ab = (T)(-dtv * dtv / (2 * lastdt));
  const bool ab2 = prm.time_step == OCU_TS_ADAMS_BASHFORD2 && lastdt > 0;
  num_steps++;
  const char *ge = std::getenv("OCU_B200_NS_GRAPH"), *ga = std::getenv("OCU_B200_GRAPHS");
  bool graphed = false;
  if (!(ge && ge[0] == '0') && !(ga && ga[0] == '0')) {
    const std::string sig = tail_env_signature();
    if (sig != tail_env) {
      drop_tail_graphs();
      tail_env = sig;
    }
    const int key = (ab2 ? 2 : 0) + (swaps & 1);
    if (stream && (tail_exec[key] || tail_seen[key] > 0)) {
      OCU_TRY(replay_tail<T>(key, dtv, ab, ab2));
      graphed = true;
    }
    tail_seen[key]++;
  }
  if (!graphed) OCU_TRY(enqueue_tail<T>(dtv, ab, ab2, nullptr));

  if (prm.time_step == OCU_TS_ADAMS_BASHFORD2) {
    // this step's derivatives become the previous ones by exchanging the buffers, where the
    // reference copies them (eqn_incompressns3d.cu:390-396).  The derivative kernels overwrite
    // every cell the update reads, except the u/v/w face layers i = nx / j = ny / k = nz, which
    // only the viscous term adds to; those faces of the velocity are set by the boundary
    // conditions after the update, so the velocity and temperature are the reference's.
    lastdt = dtv;
    swaps++;
    std::swap(dt, ldt);
    std::swap(du, ldu);
    std::swap(dv, ldv);
    std::swap(dw, ldw);
  }
  return proj.solve(prm.max_divergence);
}

// advance_one_step (eqn_incompressns3d.cu:331-399)
ocu_status NSSolver::advance_one_step(double dtv) {
  if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] advance_one_step - not initialized");
  return dtype == OCU_F64 ? step_t<double>(dtv) : step_t<float>(dtv);
}

// Equation::advance (equation.cpp:31-56)
ocu_status NSSolver::advance(double dtv) {
  if (!check_float((float)dtv)) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Equation::advance - bad dt value");
  double dtleft = dtv;
  while (dtleft > 0) {
    double maxdt;
    OCU_TRY(get_max_stable_timestep(&maxdt));
    const int subds = (int)std::ceil(dtleft / maxdt);
    const double subdt = dtleft / subds;
    ocu_status st = advance_one_step(subdt);
    if (st != OCU_OK) return st;
    dtleft -= subdt;
  }
  return OCU_OK;
}

void NSSolver::set_stream(cudaStream_t s) {
  if (!s) {
    if (!own.s) cudaStreamCreate(&own.s);
    s = own.s;
  }
  stream = s;
  proj.set_stream(s);
}

ocu_grid *NSSolver::grid(char which) {
  switch (which) {
    case 'u': return u; case 'v': return v; case 'w': return w; case 't': return t;
    case 'U': return du; case 'V': return dv; case 'W': return dw; case 'T': return dt;
    case 'p': return proj.mg ? proj.mg->s.pressure : nullptr;
    default: return nullptr;
  }
}

}  // namespace ocub
