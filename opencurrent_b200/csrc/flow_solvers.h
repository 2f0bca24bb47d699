// Projection and Navier-Stokes classes behind the ocu_project_* / ocu_ns_* entry points.
#pragma once

#include <string>

#include "mg_solver.h"

namespace ocub {

struct ProjectSolver {
  ocu_dtype dtype = OCU_F32;
  int mg_kind = -1;  // pressure solver kind (ocu_mg_kind; -1: plain, of the fields' precision)
  ocu_grid *divergence64 = nullptr;  // FP32 fields with a refinement-solved FP64 pressure: its rhs
  ocu_bc_set bc{};
  int nx = 0, ny = 0, nz = 0;
  double hx = 0, hy = 0, hz = 0;
  ocu_grid *u = nullptr, *v = nullptr, *w = nullptr;  // borrowed
  ocu_grid *divergence = nullptr;                     // owned
  ocu_mg *mg = nullptr;                               // owned pressure solver
  cudaStream_t stream = nullptr;
  bool initialized = false;

  ~ProjectSolver();
  ocu_status initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, ocu_grid *u,
                                ocu_grid *v, ocu_grid *w, const ocu_bc_set &bc);
  ocu_status solve(double tolerance);
  ocu_status solve_divergence_only();
  void set_stream(cudaStream_t s);
  template <typename T> ocu_status solve_t(double tolerance);
  ocu_status solve_f32_p64(double tolerance);
  bool p64() const { return dtype == OCU_F32 && mg_kind >= 0 && mg_kind != OCU_MG_F32; }
  template <typename T> ocu_status divergence_only_t();
};

ocu_status ns_init_layout(int nx, int ny, int nz, char which, ocu_layout *L);

// A stream the solver creates for itself (synchronised and destroyed last).
struct OwnedStream {
  cudaStream_t s = nullptr;
  ~OwnedStream() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

struct NSSolver {
  // Work runs on the caller's stream.  The legacy default stream (NULL) cannot be captured into
  // a graph, so for NULL the solver and its projection use a private blocking stream, which the
  // legacy stream orders against implicitly in both directions -- the semantics of NULL.
  // Declared before the projection so that it outlives it.
  OwnedStream own;
  ocu_dtype dtype = OCU_F32;
  ocu_ns_params prm{};
  double T_gravity = 0, T_bouyancy = 0, T_kappa = 0, T_nu = 0;
  ocu_grid *u = nullptr, *v = nullptr, *w = nullptr, *t = nullptr;
  ocu_grid *du = nullptr, *dv = nullptr, *dw = nullptr, *dt = nullptr;
  ocu_grid *ldu = nullptr, *ldv = nullptr, *ldw = nullptr, *ldt = nullptr;
  ProjectSolver proj;
  double lastdt = 0;
  int num_steps = 0;
  bool initialized = false;
  cudaStream_t stream = nullptr;
  void *scratch = nullptr;
  double *d_red = nullptr;
  double *h_red = nullptr;
  // The step's work before the projection, captured once per state as a CUDA graph and
  // replayed: state = (Adams-Bashforth form, parity of the history-buffer exchanges).  Its
  // step-dependent coefficients (dt, dt - ab, ab in the grid type) are read from d_coef, which
  // one small kernel writes before each replay.  A state's first step runs as plain launches
  // (caches of the launchers are filled outside any capture); OCU_B200_NS_GRAPH=0 or
  // OCU_B200_GRAPHS=0 (read at every step) keeps every step on plain launches.
  void *d_coef = nullptr;
  cudaGraphExec_t tail_exec[4] = {nullptr, nullptr, nullptr, nullptr};
  int tail_seen[4] = {0, 0, 0, 0};
  int tail_kernels[4] = {0, 0, 0, 0};  // kernels per replay (the library's launch count)
  int swaps = 0;
  std::string tail_env;  // the launch-shaping environment the graphs were captured under
  void drop_tail_graphs();

  ~NSSolver();
  ocu_status set_parameters(const ocu_ns_params &p, const void *iu, const void *iv, const void *iw,
                            const void *it);
  ocu_status get_max_stable_timestep(double *dt);
  ocu_status advance_one_step(double dt);
  ocu_status advance(double dt);
  void set_stream(cudaStream_t s);
  ocu_grid *grid(char which);
  template <typename T> ocu_status step_t(double dt);
  // the step up to the projection; dcoef: device coefficients (dt, dt - ab, ab) or nullptr
  template <typename T> ocu_status enqueue_tail(double dt, T ab, bool ab2, const T *dcoef);
  template <typename T> ocu_status replay_tail(int key, double dt, T ab, bool ab2);
};

}  // namespace ocub

struct ocu_project {
  ocub::ProjectSolver s;
};

struct ocu_ns {
  ocub::NSSolver s;
};
