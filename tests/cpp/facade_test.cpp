// The reference's own test flow, written against the C++ drop-in facade (include/ocu/opencurrent.h):
//   - run_all_dirichelet_test (tests/mgdoubletest.cpp:199-227): zero RHS, Dirichlet v => p == v
//   - run_neumann_test (tests/mgtest.cpp): FP32 Neumann solve reaches the tolerance
//   - ProjectTest (tests/projecttest.cpp:27-136): sine velocity field, max |div| <= 2e-4 after
//     projection
//   - NSTest-style smoke (tests/nstest.cpp): a few Boussinesq steps stay finite
// Prints "FACADE OK" and exits 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "ocu/opencurrent.h"

using namespace ocu;

static int failures = 0;
#define REQUIRE(c)                                                \
  do {                                                            \
    if (!(c)) {                                                   \
      std::printf("REQUIRE FAILED %s:%d: %s\n", __FILE__, __LINE__, #c); \
      failures++;                                                 \
      return;                                                     \
    }                                                             \
  } while (0)
#define CHECK(c)                                                  \
  do {                                                            \
    if (!(c)) {                                                   \
      std::printf("CHECK FAILED %s:%d: %s\n", __FILE__, __LINE__, #c); \
      failures++;                                                 \
    }                                                             \
  } while (0)

static void all_dirichlet(double value) {
  const int n = 32;
  Grid3DDeviceD rhs;
  REQUIRE(rhs.init(n, n, n, 1, 1, 1));
  CHECK(rhs.clear_zero());
  Sol_MultigridPressure3DDeviceD solver;
  BoundaryCondition d;
  d.type = BC_DIRICHELET;
  d.value = (float)value;
  solver.bc = BoundaryConditionSet(d);
  REQUIRE(solver.initialize_storage(n, n, n, 4.0 / n, 4.0 / n, 4.0 / n, &rhs));
  Grid3DHostD init;
  init.init_congruent(solver.pressure());
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++) init.at(i, j, k) = 0.5 - std::fmod(0.618033988749 * (i * n * n + j * n + k), 1.0);
  CHECK(solver.pressure().copy_all_data(init));
  double residual = 0;
  CHECK(solver.solve(residual, 1e-8, 15));
  CHECK(residual < 1e-8);
  double mx = 0, mn = 0;
  CHECK(solver.pressure().reduce_max(mx));
  CHECK(solver.pressure().reduce_min(mn));
  CHECK(std::fabs(mx - value) < 1e-7 && std::fabs(mn - value) < 1e-7);
}

static void neumann_fp32() {
  const int n = 64;
  Grid3DHostF h;
  h.init(n, n, n, 1, 1, 1);
  double mean = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++) {
        const double x = (i + 0.5) / n, y = (j + 0.5) / n, z = (k + 0.5) / n;
        mean += std::cos(M_PI * x) * std::cos(2 * M_PI * y) * std::cos(3 * M_PI * z);
      }
  mean /= (double)n * n * n;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++) {
        const double x = (i + 0.5) / n, y = (j + 0.5) / n, z = (k + 0.5) / n;
        h.at(i, j, k) = (float)(std::cos(M_PI * x) * std::cos(2 * M_PI * y) * std::cos(3 * M_PI * z) - mean);
      }
  Grid3DDeviceF rhs;
  REQUIRE(rhs.init_congruent(h));
  CHECK(rhs.copy_all_data(h));
  Sol_MultigridPressure3DDeviceF solver;
  BoundaryCondition neu;
  neu.type = BC_NEUMANN;
  solver.bc = BoundaryConditionSet(neu);
  REQUIRE(solver.initialize_storage(n, n, n, 1.0 / n, 1.0 / n, 1.0 / n, &rhs));
  double residual = 0;
  CHECK(solver.solve(residual, 1e-4, 10));
  CHECK(residual < 1e-4);
  CHECK(!solver.any_error());
}

static void projection() {
  const int nx = 64, ny = 32, nz = 32;
  const double hx = .5, hy = .5, hz = 1;
  Grid3DDeviceF u, v, w;
  REQUIRE(u.init(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1));
  REQUIRE(v.init(nx, ny + 1, nz, 1, 1, 1, 1, 0, 1));
  REQUIRE(w.init(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0));
  Grid3DHostF hu, hv, hw;
  hu.init_congruent(u);
  hv.init_congruent(v);
  hw.init_congruent(w);
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        hu.at(i, j, k) = std::sin(((float)k) / nz * 4 * M_PI) + std::sin(((float)j) / ny * 4 * M_PI);
        hv.at(i, j, k) = std::sin(((float)k) / nz * 8 * M_PI) + std::sin(((float)i) / nx * 6 * M_PI);
        hw.at(i, j, k) = std::cos(((float)j) / ny * 8 * M_PI) + std::sin(((float)k) / nz * 6 * M_PI);
      }
  CHECK(u.copy_all_data(hu));
  CHECK(v.copy_all_data(hv));
  CHECK(w.copy_all_data(hw));
  Sol_ProjectDivergence3DDeviceF project;
  BoundaryCondition closed;
  closed.type = BC_FORCED_INFLOW_VARIABLE_SLIP;
  BoundaryCondition periodic;
  periodic.type = BC_PERIODIC;
  project.bc = BoundaryConditionSet(periodic);
  project.bc.zpos = closed;
  project.bc.zneg = closed;
  CHECK(apply_3d_mac_boundary_conditions_level1(u, v, w, project.bc, hx, hy, hz));
  CHECK(project.initialize_storage(nx, ny, nz, hx, hy, hz, &u, &v, &w));
  CHECK(project.solve(2e-4));
  CHECK(project.solve_divergence_only());
  float max_div = 1;
  CHECK(project.divergence().reduce_maxabs(max_div));
  CHECK(max_div <= 2e-4f);
}

// projectdoubletest.cpp-style check of the mixed class: max |div| <= 1e-10 after an FP64
// projection with the mixed pressure solver, both algorithms
static void projection_mixed(bool reference_algorithm) {
  const int nx = 32, ny = 32, nz = 32;
  const double hx = 1.0 / nx, hy = 1.0 / ny, hz = 1.0 / nz;
  Grid3DDeviceD u, v, w;
  REQUIRE(u.init(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1));
  REQUIRE(v.init(nx, ny + 1, nz, 1, 1, 1, 1, 0, 1));
  REQUIRE(w.init(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0));
  Grid3DHostD hu, hv, hw;
  hu.init_congruent(u);
  hv.init_congruent(v);
  hw.init_congruent(w);
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        hu.at(i, j, k) = std::sin(((double)k) / nz * 4 * M_PI) + std::cos(((double)j) / ny * 2 * M_PI);
        hv.at(i, j, k) = std::sin(((double)i) / nx * 6 * M_PI);
        hw.at(i, j, k) = std::cos(((double)j) / ny * 8 * M_PI) * std::sin(((double)i) / nx * 2 * M_PI);
      }
  CHECK(u.copy_all_data(hu));
  CHECK(v.copy_all_data(hv));
  CHECK(w.copy_all_data(hw));
  Sol_ProjectDivergenceMixed3DDeviceD project;
  if (reference_algorithm) project.use_reference_algorithm();
  BoundaryCondition closed;
  closed.type = BC_FORCED_INFLOW_VARIABLE_SLIP;
  project.bc = BoundaryConditionSet(closed);
  CHECK(project.initialize_storage(nx, ny, nz, hx, hy, hz, &u, &v, &w));
  CHECK(project.solve(1e-10));
  CHECK(project.solve_divergence_only());
  double max_div = 1;
  CHECK(project.divergence().reduce_maxabs(max_div));
  CHECK(max_div <= 1e-10);
}

// failure paths through the facade: max_iter exhausted (false, the reference's sticky error
// stays clear on the solver, as Sol_MultigridPressure3DBase::solve sets none), a projection whose
// pressure solve fails (false, any_error() set), both usable afterwards
static void failure_paths() {
  const int n = 32;
  Grid3DDeviceF rhs;
  REQUIRE(rhs.init(n, n, n, 1, 1, 1));
  Grid3DHostF h;
  h.init_congruent(rhs);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++) h.at(i, j, k) = std::cos(M_PI * (i + .5) / n) * std::cos(2 * M_PI * (k + .5) / n);
  CHECK(rhs.copy_all_data(h));
  Sol_MultigridPressure3DDeviceF solver;
  BoundaryCondition neumann;
  neumann.type = BC_NEUMANN;
  solver.bc = BoundaryConditionSet(neumann);
  REQUIRE(solver.initialize_storage(n, n, n, 1.0 / n, 1.0 / n, 1.0 / n, &rhs));
  double residual = 0;
  CHECK(!solver.solve(residual, 1e-30, 2));
  CHECK(std::isfinite(residual) && residual > 0);
  CHECK(!solver.any_error());
  CHECK(solver.solve(residual, 1e-4, 20));

  const int nx = 16, ny = 16, nz = 16;
  Grid3DDeviceF u, v, w;
  REQUIRE(u.init(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1));
  REQUIRE(v.init(nx, ny + 1, nz, 1, 1, 1, 1, 0, 1));
  REQUIRE(w.init(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0));
  u.clear(1.0f);
  v.clear(-0.5f);
  w.clear(0.25f);
  Sol_ProjectDivergence3DDeviceF project;
  BoundaryCondition closed;
  closed.type = BC_FORCED_INFLOW_VARIABLE_SLIP;
  project.bc = BoundaryConditionSet(closed);
  CHECK(project.initialize_storage(nx, ny, nz, 1.0 / nx, 1.0 / ny, 1.0 / nz, &u, &v, &w));
  CHECK(!project.solve(1e-30));
  CHECK(project.any_error());
  CHECK(project.solve(1e-3));
  CHECK(!project.any_error());
}

static void ns_smoke() {
  Eqn_IncompressibleNS3DParamsD params;
  params.init_grids(32, 32, 16);
  params.hx = params.hy = params.hz = 1.0 / 16;
  BoundaryCondition periodic, wall, hot, cold;
  periodic.type = BC_PERIODIC;
  wall.type = BC_FORCED_INFLOW_VARIABLE_SLIP;
  wall.aux_value = 1;
  hot.type = BC_DIRICHELET;
  hot.value = 1;
  cold.type = BC_DIRICHELET;
  params.flow_bc = BoundaryConditionSet(periodic);
  params.flow_bc.zpos = wall;
  params.flow_bc.zneg = wall;
  params.temp_bc = BoundaryConditionSet(periodic);
  params.temp_bc.zpos = cold;
  params.temp_bc.zneg = hot;
  params.vertical_direction = DIR_ZPOS;
  params.gravity = -1;
  params.bouyancy = 2000;
  params.viscosity = 1;
  params.thermal_diffusion = 1;
  params.max_divergence = 1e-9;
  for (int i = 0; i < 32; i++)
    for (int j = 0; j < 32; j++)
      for (int k = 0; k < 16; k++)
        params.init_temp.at(i, j, k) = 1 - (k + .5) / 16 + 1e-3 * std::sin(0.7 * i + 1.3 * j);
  Eqn_IncompressibleNS3DD eqn;
  REQUIRE(eqn.set_parameters(params));
  for (int s = 0; s < 5; s++) CHECK(eqn.advance_one_step(eqn.get_max_stable_timestep()));
  double tmax = 0;
  CHECK(eqn.get_temperature().reduce_maxabs(tmax));
  CHECK(std::isfinite(tmax) && tmax <= 1.0 + 1e-2);
  CHECK(eqn.num_steps() == 5);
}

// Sol_PCGPressure3DDevice: a variable coefficient, multigrid-preconditioned CG to 1e-8 (FP64)
static void pcg(PreconditionerType pc) {
  const int n = 16;
  const float h = 1.0f / n;
  Grid3DDeviceD rhs, coef;
  REQUIRE(rhs.init(n, n, n, 1, 1, 1));
  REQUIRE(coef.init_congruent(rhs));
  Grid3DHostD hr, hc;
  REQUIRE(hr.init_congruent(rhs));
  REQUIRE(hc.init_congruent(rhs));
  double mean = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++) {
        hr.at(i, j, k) = std::sin(6.28318530718 * (i + 0.5) / n) * std::cos(3.14159265359 * (k + 0.5) / n) + 0.01 * j;
        mean += hr.at(i, j, k);
        hc.at(i, j, k) = 1.0 + 0.5 * std::sin(6.28318530718 * (j + 0.5) / n);
      }
  mean /= (double)n * n * n;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++) hr.at(i, j, k) -= mean;
  CHECK(rhs.copy_all_data(hr));
  CHECK(coef.copy_all_data(hc));
  Sol_PCGPressure3DDeviceD solver;
  BoundaryCondition per, neu;
  per.type = BC_PERIODIC;
  neu.type = BC_NEUMANN;
  solver.bc = BoundaryConditionSet(neu);
  solver.bc.xpos = solver.bc.xneg = per;
  solver.preconditioner = pc;
  REQUIRE(solver.initialize_storage(n, n, n, h, h, h, &rhs, &coef));
  double residual = 0;
  CHECK(solver.solve(residual, 1e-8, 300));
  CHECK(residual < 1e-8);
  CHECK(!solver.any_error());
  // max_iter too small: solve() returns false, as the reference does
  double r2 = 0;
  solver.pressure().clear_zero();
  CHECK(!solver.solve(r2, 1e-14, 2));
}

// NetCDFGrid3DWriter / Reader: a cell-centred and a u-face grid over two time levels, read back
static void netcdf_round_trip() {
  const char *path = "facade_test_grids.nc";
  Grid3DHostF t;
  Grid3DHostD u;
  REQUIRE(t.init(5, 4, 3, 1, 1, 1));
  REQUIRE(u.init(6, 4, 3, 1, 1, 1));
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 3; k++) {
        if (i < 5) t.at(i, j, k) = (float)(i * 100 + j * 10 + k);
        u.at(i, j, k) = 0.5 * i - 0.25 * j + 0.125 * k;
      }
  NetCDFGrid3DWriter w;
  REQUIRE(w.open(path, 5, 4, 3, 0.2f, 0.25f, 1.0f / 3));
  CHECK(w.define_variable("temp", NC_FLOAT, GS_CENTER_POINT));
  CHECK(w.define_variable("u", NC_DOUBLE, GS_U_FACE));
  CHECK(w.add_data("temp", t, 0));
  size_t level = 0;
  CHECK(w.add_time_level(0.5f, level) && level == 1);
  CHECK(w.add_data("u", u, 1));
  CHECK(w.close());
  NetCDFGrid3DReader r;
  REQUIRE(r.open(path));
  CHECK(r.nx() == 5 && r.ny() == 4 && r.nz() == 3 && r.num_time_levels() == 2 && r.get_time(1) == 0.5f);
  CHECK(r.list_variables().size() == 2);
  int nx = 0, ny = 0, nz = 0;
  CHECK(r.variable_size("u", nx, ny, nz) && nx == 6);
  Grid3DHostF t2;
  Grid3DHostD u2;
  REQUIRE(t2.init(5, 4, 3, 1, 1, 1));
  REQUIRE(u2.init(6, 4, 3, 1, 1, 1));
  CHECK(r.read_variable("temp", t2, 0));
  CHECK(r.read_variable("u", u2, 1));
  CHECK(t2.at(4, 3, 2) == 432.0f && u2.at(5, 0, 1) == 2.625);
  r.close();
  std::remove(path);
}

// Sol_MultigridPressure3DDeviceCo: two images of a 64x32x32 Neumann problem on one device give,
// after the same FMG + V-cycles, the single-image solver's pressure bit for bit.
static void co_array_mg() {
  const int nx = 64, ny = 32, nz = 32, N = 2, nxl = nx / N;
  Grid3DHostD whole, part[N];
  REQUIRE(whole.init(nx, ny, nz, 1, 1, 1));
  for (int q = 0; q < N; q++) REQUIRE(part[q].init(nxl, ny, nz, 1, 1, 1));
  double mean = 0;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) mean += whole.at(i, j, k) = std::sin(0.3 * i + 0.2 * j) * std::cos(0.1 * k + 0.05 * i);
  mean /= (double)nx * ny * nz;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        whole.at(i, j, k) -= mean;
        part[i / nxl].at(i % nxl, j, k) = whole.at(i, j, k);
      }
  Grid3DDeviceD rhs, rhs_part[N];
  REQUIRE(rhs.init(nx, ny, nz, 1, 1, 1));
  REQUIRE(rhs.copy_all_data(whole));
  Grid3DDeviceD *parts[N];
  for (int q = 0; q < N; q++) {
    REQUIRE(rhs_part[q].init(nxl, ny, nz, 1, 1, 1));
    REQUIRE(rhs_part[q].copy_all_data(part[q]));
    parts[q] = &rhs_part[q];
  }
  BoundaryCondition neu;
  neu.type = BC_NEUMANN;
  Sol_MultigridPressure3DDeviceD one;
  one.bc = BoundaryConditionSet(neu);
  REQUIRE(one.initialize_storage(nx, ny, nz, 1.0 / nx, 1.0 / ny, 1.0 / nz, &rhs));
  Sol_MultigridPressure3DDeviceCo<double> co("p", N);
  co.bc = BoundaryConditionSet(neu);
  co.grid_size_for_cutoff = 512;
  REQUIRE(co.initialize_storage(nxl, ny, nz, 1.0 / nx, 1.0 / ny, 1.0 / nz, parts));
  CHECK(co.num_images() == N && co.cutoff_level() == 3);
  CHECK(one.run_fmg(1) && co.run_fmg(1));
  CHECK(one.run_vcycles(2) && co.run_vcycles(2));
  Grid3DHostD a, b;
  REQUIRE(a.init_congruent(one.pressure()));
  REQUIRE(a.copy_all_data(one.pressure()));
  int differ = 0;
  for (int q = 0; q < N; q++) {
    REQUIRE(b.init_congruent(co.co_pressure(q)));
    REQUIRE(b.copy_all_data(co.co_pressure(q)));
    for (int i = 0; i < nxl; i++)
      for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) differ += std::memcmp(&a.at(q * nxl + i, j, k), &b.at(i, j, k), sizeof(double)) != 0;
  }
  CHECK(differ == 0);
  double res = 0;
  CHECK(co.solve(res, 1e-9, 15) && res < 1e-9);
}

int main() {
  all_dirichlet(0.0);
  all_dirichlet(0.5);
  neumann_fp32();
  projection();
  projection_mixed(false);
  projection_mixed(true);
  failure_paths();
  ns_smoke();
  pcg(PRECOND_MULTIGRID);
  pcg(PRECOND_JACOBI);
  netcdf_round_trip();
  co_array_mg();
  if (failures) {
    std::printf("FACADE FAILED (%d)\n", failures);
    return 1;
  }
  std::printf("FACADE OK\n");
  return 0;
}
