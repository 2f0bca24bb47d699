/*
 * ocu_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, CPU-only restatement of OpenCurrent's projection-step hot path, used as the
 * parity checker for the CUDA library in opencurrent_b200/.  Only tests/, the smoke check
 * in __graft_entry__.py and the CPU-baseline leg of bench.py may load it; the product path
 * never links it.
 *
 * Every function restates the reference's arithmetic in the reference's operation order,
 * with floating-point contraction disabled (-ffp-contract=off), so that a CUDA kernel built
 * with --fmad=false and the same operation order matches it bit for bit.  Each function's
 * comment names the reference file:line it follows.  Suffix _f = float, _d = double.
 *
 * Parity pin: the oracle is checked against the reference's own known-answer tests
 * (tests/mgtest.cpp, mgdoubletest.cpp, projecttest.cpp, advection3d*test.cpp,
 * rayleigh.cpp) in tests/test_oracle_*.py, and against the reference device solver compiled
 * from its own sources (oracle/build_ref.sh -> oracle/_ref/) in the GPU test suite.
 */
#ifndef OCU_ORACLE_H
#define OCU_ORACLE_H

#include "../include/ocu_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Grid3DDevice<T>::init layout rule (ocustorage/grid3ddev.cu:358-400). */
void orc_layout(int nx, int ny, int nz, int gx, int gy, int gz, int padx, int pady, int padz,
                ocu_layout *out);

/* Multigrid level count (ocuequation/sol_mgpressure3d.cpp:67-92). */
int orc_num_levels(int nx, int ny, int nz);
/* Yavneh's red-black SOR omega (ocuequation/sol_mgpressure3d.cpp:94-109). */
double orc_optimal_omega(double fx, double fy, double fz);

#define ORC_DECLARE(T, S)                                                                         \
  int orc_bc_level1##S(T *p, const ocu_layout *L, const ocu_bc_set *bc, double hx, double hy,    \
                       double hz);                                                                \
  int orc_bc_nocorners_dev##S(T *p, const ocu_layout *L, const ocu_bc_set *bc, double hx,        \
                              double hy, double hz);                                              \
  int orc_bc_nocorners_host##S(T *p, const ocu_layout *L, const ocu_bc_set *bc, double hx,       \
                               double hy, double hz);                                             \
  int orc_mac_bc_level1##S(T *u, T *v, T *w, const ocu_layout *Lu, int nx, int ny, int nz,       \
                           const ocu_bc_set *bc, double hx, double hy, double hz);               \
  double orc_reduce##S(const T *p, const ocu_layout *L, int op);                                  \
  void orc_lincomb1##S(T *res, const ocu_layout *L, double a1, const T *g1);                      \
  void orc_lincomb2##S(T *res, const ocu_layout *L, double a1, const T *g1, double a2,            \
                       const T *g2);                                                              \
  void orc_divergence##S(const T *u, const T *v, const T *w, T *div, const ocu_layout *L, int nx, \
                         int ny, int nz, double hx, double hy, double hz);                        \
  void orc_gradient##S(T *u, T *v, T *w, const T *phi, const ocu_layout *L, int nx, int ny,       \
                       int nz, double hx, double hy, double hz, double coefficient);              \
  void orc_laplacian##S(const T *phi, T *dphidt, const ocu_layout *L, int nx, int ny, int nz,     \
                        double hx, double hy, double hz, double coefficient);                     \
  void orc_advect_self##S(const T *u, const T *v, const T *w, T *dudt, T *dvdt, T *dwdt,          \
                          const ocu_layout *L, int nx, int ny, int nz, double hx, double hy,      \
                          double hz, int interp);                                                 \
  void orc_advect_passive##S(const T *u, const T *v, const T *w, const T *phi, T *dphidt,        \
                             const ocu_layout *L, int nx, int ny, int nz, double hx, double hy,   \
                             double hz, int interp);                                              \
  void orc_thermal_force##S(T *dvdt, double coefficient, const T *temp, const ocu_layout *L,      \
                            int nbr_stride, int nx, int ny, int nz);                              \
  void orc_pcg_laplacian##S(T *dst, const T *src, const T *coef, const ocu_layout *L, double fxh, \
                            double fyh, double fzh);                                              \
  void orc_pcg_diag##S(T *dst, const T *src, const T *coef, const ocu_layout *L, double fxh,      \
                       double fyh, double fzh);                                                   \
  double orc_pcg_dot##S(const T *a, const T *b, const ocu_layout *L);

ORC_DECLARE(float, _f)
ORC_DECLARE(double, _d)

/* ------------------------------------------------------------------------------------------
 * Multigrid pressure solver (Sol_MultigridPressure3DDevice<T>, ocuequation/sol_mgpressure3d*).
 * The oracle owns the coarse levels and u0 (the "pressure" grid, congruent with rhs); it
 * borrows the rhs buffer exactly like the reference (sol_mgpressure3ddev.cu:418).
 * ---------------------------------------------------------------------------------------- */
typedef struct orc_mg_params {
  ocu_bc_set bc;
  int nu1, nu2;
  int convergence;
  int make_symmetric_operator;
  int disable_relax_on_host;
} orc_mg_params;

typedef struct orc_mg orc_mg;

/* dtype: OCU_F32 or OCU_F64.  rhs must have ghost >= 1; its layout is used for u0/r0. */
orc_mg *orc_mg_create(int dtype, const orc_mg_params *prm, int nx, int ny, int nz, double hx,
                      double hy, double hz, void *rhs, const ocu_layout *rhs_layout);
void orc_mg_destroy(orc_mg *mg);
void orc_mg_set_params(orc_mg *mg, const orc_mg_params *prm);
/* Base::solve (sol_mgpressure3d.cpp:332-370). Returns 1 on convergence. */
int orc_mg_solve(orc_mg *mg, double *residual, double tolerance, int max_iter);
int orc_mg_run_vcycles(orc_mg *mg, int count);  /* sol_mgpressure3d.cpp:372-384 */
int orc_mg_run_fmg(orc_mg *mg, int count);      /* sol_mgpressure3d.cpp:386-398 */
int orc_mg_num_levels(const orc_mg *mg);
/* Level operations (relax, one colour sweep, restrict_residuals, prolong+BC) on the interface
 * hierarchy (core 0) or the FP32 hierarchy of a mixed solver (core 1). */
int orc_mg_relax(orc_mg *mg, int core, int level, int iterations, int order);
int orc_mg_relax_sweep(orc_mg *mg, int core, int level, int color);
int orc_mg_restrict_residuals(orc_mg *mg, int core, int fine, int coarse, double *l2, double *linf);
int orc_mg_prolong(orc_mg *mg, int core, int coarse, int fine);
/* which: 'u', 'b', 'r'.  Returns the level's buffer (host memory owned by the oracle). */
void *orc_mg_grid(orc_mg *mg, char which, int level, ocu_layout *layout_out);
int orc_mg_vcycles(const orc_mg *mg); /* fine-level cycles run by the last do_fmg */
double orc_mg_omega(const orc_mg *mg);

/* Reference mixed solver: FP32 FMG warm start then FP64 FMG
 * (ocuequation/sol_mgpressuremixed3ddevd.cpp:79-138).  rhs is a double grid. */
orc_mg *orc_mgmixed_create(const orc_mg_params *prm, int nx, int ny, int nz, double hx,
                           double hy, double hz, double *rhs, const ocu_layout *rhs_layout);

/* FP32-in-FP64 iterative refinement (the B200 build's mixed algorithm; no reference
 * counterpart).  inner_cycles = FP32 fine-level V-cycles per FMG correction solve. */
orc_mg *orc_mgir_create(const orc_mg_params *prm, int nx, int ny, int nz, double hx, double hy,
                        double hz, double *rhs, const ocu_layout *rhs_layout, int inner_cycles);
int orc_mgir_outer_iterations(const orc_mg *mg);

/* ------------------------------------------------------------------------------------------
 * Projection (Sol_ProjectDivergence3DDevice<T>, ocuequation/sol_project3ddev.cu:28-135).
 * Borrows u, v, w (MAC grids of one common layout); owns divergence + pressure solver.
 * ---------------------------------------------------------------------------------------- */
typedef struct orc_project orc_project;
orc_project *orc_project_create(int dtype, const ocu_bc_set *bc, int nx, int ny, int nz,
                                double hx, double hy, double hz, void *u, void *v, void *w,
                                const ocu_layout *mac_layout);
/* kind 0/1: FP32/FP64; 2: Sol_ProjectDivergenceMixed3DDeviceD (reference mixed pressure
 * solver, sol_projectmixed3d.cu:48-91); 3: the same class with the FP32-in-FP64 refinement
 * solver (inner_cycles per correction).  Kinds 2 and 3 take double grids. */
orc_project *orc_project_create_kind(int kind, const ocu_bc_set *bc, int nx, int ny, int nz,
                                     double hx, double hy, double hz, void *u, void *v, void *w,
                                     const ocu_layout *mac_layout, int inner_cycles);
void orc_project_destroy(orc_project *p);
int orc_project_solve(orc_project *p, double tolerance);
int orc_project_solve_divergence_only(orc_project *p);
void *orc_project_divergence(orc_project *p);
orc_mg *orc_project_pressure_solver(orc_project *p);

/* ------------------------------------------------------------------------------------------
 * Preconditioned conjugate gradients (Sol_PCGPressure3DDevice<T>,
 * ocuequation/sol_pcgpressure3d.cu:289-654): L p = rhs with L = -div(c grad), c a cell
 * coefficient grid; preconditioner none, Jacobi, multigrid (FMG or V-cycles on the constant-
 * coefficient operator, sign flipped) or BFBT (multigrid then Jacobi).  Borrows rhs and
 * coefficient (one layout, ghost >= 1); owns the pressure and the CG vectors.
 * ---------------------------------------------------------------------------------------- */
typedef struct orc_pcg_params {
  ocu_bc_set bc;
  int convergence;       /* OCU_CONVERGENCE_L2 (default) or _LINF: which norm solve() returns */
  int preconditioner;    /* ocu_precond (default OCU_PRECOND_BFBT) */
  int multigrid_cycles;  /* default 2 */
  int multigrid_use_fmg; /* default 1 */
} orc_pcg_params;
typedef struct orc_pcg orc_pcg;
/* hx, hy, hz are rounded to float (the reference's initialize_storage takes float). */
orc_pcg *orc_pcg_create(int dtype, const orc_pcg_params *prm, int nx, int ny, int nz, double hx, double hy,
                        double hz, void *rhs, void *coefficient, const ocu_layout *layout);
void orc_pcg_destroy(orc_pcg *p);
/* solve (sol_pcgpressure3d.cu:571-601); returns 1 when converged, *residual the chosen norm. */
int orc_pcg_solve(orc_pcg *p, double *residual, double tolerance, int max_iter);
void *orc_pcg_pressure(orc_pcg *p);
int orc_pcg_iterations(const orc_pcg *p);

/* ------------------------------------------------------------------------------------------
 * Incompressible Navier-Stokes / Boussinesq (Eqn_IncompressibleNS3D<T>,
 * ocuequation/eqn_incompressns3d.cu:164-399, equation.cpp:31-56).
 * ---------------------------------------------------------------------------------------- */
typedef struct orc_ns_params {
  int nx, ny, nz;
  double hx, hy, hz;
  double max_divergence;
  ocu_bc_set temp_bc;
  ocu_bc_set flow_bc;
  int vertical_direction;
  double gravity;           /* stored as T by the equation */
  double bouyancy;          /* stored as T */
  double thermal_diffusion; /* stored as T */
  double viscosity;         /* stored as T */
  int advection_scheme;
  int time_step;
  double cfl_factor;
} orc_ns_params;

typedef struct orc_ns orc_ns;
/* init_* are host grids in the layout produced by Eqn_IncompressibleNS3DParams::init_grids
 * (eqn_incompressns3d.h:75-83): u (nx+1,ny,nz) pad (0,1,1), v pad (1,0,1), w pad (1,1,0),
 * temp pad (1,1,1); all congruent. */
orc_ns *orc_ns_create(int dtype, const orc_ns_params *prm, const void *init_u,
                      const void *init_v, const void *init_w, const void *init_temp);
void orc_ns_destroy(orc_ns *ns);
double orc_ns_get_max_stable_timestep(orc_ns *ns);
int orc_ns_advance_one_step(orc_ns *ns, double dt);
int orc_ns_advance(orc_ns *ns, double dt);
/* which: 'u','v','w','t' (state) or 'U','V','W','T' (time derivatives), 'p' (pressure). */
void *orc_ns_grid(orc_ns *ns, char which);
void orc_ns_layout(orc_ns *ns, ocu_layout *out);
void orc_ns_set_omp_threads(int n);

#ifdef __cplusplus
}
#endif

#endif /* OCU_ORACLE_H */
