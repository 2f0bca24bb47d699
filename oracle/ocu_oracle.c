/*
 * ocu_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of OpenCurrent's projection-step
 * hot path (see ocu_oracle.h).  Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include "ocu_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { ORC_RO_RED_BLACK = 0, ORC_RO_BLACK_RED = 1, ORC_RO_SYMMETRIC = 2 };

/* check_float takes a float (ocuutil/float_routines.h:33-51): a double beyond FLT_MAX fails. */
static int orc_check_float(float f) { return isfinite(f) ? 1 : 0; }

static double orc_min3(double a, double b, double c)
{
  return a < b ? (a < c ? a : c) : (b < c ? b : c);
}

static int orc_bc_is(const ocu_bc *b, int t1, int t2, int t3, int t4)
{
  return b->type == t1 || b->type == t2 || b->type == t3 || b->type == t4;
}

/* BoundaryConditionSet::check_type(BC_NONE, BC_PERIODIC, BC_DIRICHELET, BC_NEUMANN) */
static int orc_bc_check_scalar(const ocu_bc_set *s)
{
  const ocu_bc *f[6] = {&s->xpos, &s->xneg, &s->ypos, &s->yneg, &s->zpos, &s->zneg};
  int i;
  for (i = 0; i < 6; i++)
    if (!orc_bc_is(f[i], OCU_BC_NONE, OCU_BC_PERIODIC, OCU_BC_DIRICHELET, OCU_BC_NEUMANN)) return 0;
  return 1;
}

/* check_type(BC_NONE, BC_PERIODIC, BC_FORCED_INFLOW_VARIABLE_SLIP) */
static int orc_bc_check_mac(const ocu_bc_set *s)
{
  const ocu_bc *f[6] = {&s->xpos, &s->xneg, &s->ypos, &s->yneg, &s->zpos, &s->zneg};
  int i;
  for (i = 0; i < 6; i++)
    if (!orc_bc_is(f[i], OCU_BC_NONE, OCU_BC_PERIODIC, OCU_BC_FORCED_INFLOW_VARIABLE_SLIP, -1)) return 0;
  return 1;
}

static int orc_any_periodic(const ocu_bc_set *s)
{
  return s->xpos.type == OCU_BC_PERIODIC || s->xneg.type == OCU_BC_PERIODIC ||
         s->ypos.type == OCU_BC_PERIODIC || s->yneg.type == OCU_BC_PERIODIC ||
         s->zpos.type == OCU_BC_PERIODIC || s->zneg.type == OCU_BC_PERIODIC;
}

/* BoundaryConditionSet::make_homogeneous (boundary_condition.h:88-101) */
static void orc_make_homogeneous(ocu_bc_set *s)
{
  s->xpos.value = s->xpos.aux_value = 0;
  s->xneg.value = s->xneg.aux_value = 0;
  s->ypos.value = s->ypos.aux_value = 0;
  s->yneg.value = s->yneg.aux_value = 0;
  s->zpos.value = s->zpos.aux_value = 0;
  s->zneg.value = s->zneg.aux_value = 0;
}

/* bc_diag_mod (sol_mgpressure3d.cpp:49-64) */
static double orc_bc_diag_mod(const ocu_bc *b, double factor)
{
  if (b->type == OCU_BC_DIRICHELET) return factor;
  if (b->type == OCU_BC_NEUMANN) return -factor;
  return 0;
}

void orc_layout(int nx, int ny, int nz, int gx, int gy, int gz, int padx, int pady, int padz,
                ocu_layout *L)
{
  int pre_padding = 16 - gz;
  memset(L, 0, sizeof(*L));
  L->nx = nx; L->ny = ny; L->nz = nz;
  L->gx = gx; L->gy = gy; L->gz = gz;
  L->pnx = nx + 2 * gx + padx;
  L->pny = ny + 2 * gy + pady;
  L->pnz = nz + 2 * gz + padz;
  if (L->pnz & 15) L->pnz = ((L->pnz >> 4) + 1) << 4;
  L->ystride = L->pnz;
  L->xstride = L->pnz * L->pny;
  L->allocated = (long long)L->xstride * L->pnx + pre_padding;
  L->shift = (long long)gx * L->xstride + (long long)gy * L->pnz + gz + pre_padding;
}

int orc_num_levels(int nx_val, int ny_val, int nz_val)
{
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

double orc_optimal_omega(double fx, double fy, double fz)
{
  double f_min = orc_min3(fx, fy, fz);
  double c_max = (1.0 - f_min / (fx + fy + fz));
  double c_max_sqr = c_max * c_max;
  return 2.0 / (1.0 + sqrt(1.0f - c_max_sqr));
}

#define T float
#define S _f
#include "oracle_body.inc"
#undef T
#undef S

#define T double
#define S _d
#include "oracle_body.inc"
#undef T
#undef S

/* ------------------------------------------------------------------------------------------
 * Multigrid driver: Sol_MultigridPressure3DBase (sol_mgpressure3d.cpp:113-398) with the
 * virtual level operations dispatched to the float or double core, which is how the reference
 * mixed solver switches precision (sol_mgpressuremixed3ddevd.cpp:29-70).
 * ---------------------------------------------------------------------------------------- */
enum { ORC_KIND_F = 0, ORC_KIND_D = 1, ORC_KIND_MIXED = 2, ORC_KIND_IR = 3 };

struct orc_mg {
  int kind;
  orc_mg_params prm;
  int num_levels;
  int (*dim)[3];
  mgcore_f *cf;
  mgcore_d *cd;
  int double_mode;
  float *rhs_f; /* mixed / IR: float rhs owned here */
  int last_vcycles;
  int inner_cycles;
  int outer_iters;
};

static void mg_relax(orc_mg *m, int l, int it, int order)
{
  if (m->double_mode) core_relax_d(m->cd, l, it, order); else core_relax_f(m->cf, l, it, order);
}
static void mg_clear_zero(orc_mg *m, int l)
{
  if (m->double_mode) core_clear_zero_d(m->cd, l); else core_clear_zero_f(m->cf, l);
}
static void mg_apply_bc(orc_mg *m, int l)
{
  if (m->double_mode) core_apply_bc_d(m->cd, l); else core_apply_bc_f(m->cf, l);
}
static void mg_restrict_residuals(orc_mg *m, int f, int c, double *l2, double *linf)
{
  if (m->double_mode) core_restrict_residuals_d(m->cd, f, c, l2, linf);
  else core_restrict_residuals_f(m->cf, f, c, l2, linf);
}
static void mg_prolong(orc_mg *m, int c, int f)
{
  if (m->double_mode) core_prolong_bc_d(m->cd, c, f); else core_prolong_bc_f(m->cf, c, f);
}

static int mg_coarse_iters(const orc_mg *m)
{
  int cl = m->num_levels - 1;
  int a = m->dim[cl][0] * m->dim[cl][1], b = m->dim[cl][1] * m->dim[cl][2], c = m->dim[cl][0] * m->dim[cl][2];
  int mx = a > b ? (a > c ? a : c) : (b > c ? b : c);
  return mx / 2;
}

static double mg_pick(int conv, double l2, double linf)
{
  return (conv & OCU_CONVERGENCE_CRITERIA_L2) ? l2 : (conv & OCU_CONVERGENCE_CRITERIA_LINF) ? linf : 1e20;
}

/* do_fmg (sol_mgpressure3d.cpp:113-251) */
static int mg_do_fmg(orc_mg *m, double tolerance, int max_iter, double *rl2, double *rlinf)
{
  const int conv = m->prm.convergence;
  const int coarse_level = m->num_levels - 1;
  int level, fine_level, i_cyc, num_vcyc = 0;
  double orig_l2 = 0, orig_linf = 0, orig_error;
  *rl2 = *rlinf = 0;
  m->last_vcycles = 0;
  mg_apply_bc(m, 0);
  mg_restrict_residuals(m, 0, 0, (conv & OCU_CONVERGENCE_CALC_L2) ? &orig_l2 : 0,
                        (conv & OCU_CONVERGENCE_CALC_LINF) ? &orig_linf : 0);
  orig_error = mg_pick(conv, orig_l2, orig_linf);
  if (orig_error < tolerance) {
    if (conv & OCU_CONVERGENCE_CALC_L2) *rl2 = orig_l2;
    if (conv & OCU_CONVERGENCE_CALC_LINF) *rlinf = orig_linf;
    return 1;
  }
  for (level = 0; level < m->num_levels - 1; level++) {
    mg_clear_zero(m, level + 1);
    mg_apply_bc(m, level + 1);
    mg_restrict_residuals(m, level, level + 1, 0, 0);
  }
  for (fine_level = m->num_levels - 1; fine_level >= 0; fine_level--) {
    int level_ncyc = (fine_level == 0) ? max_iter + 1 : 1;
    for (i_cyc = 0; i_cyc < level_ncyc; i_cyc++) {
      if (fine_level == 0) num_vcyc++;
      for (level = fine_level; level < coarse_level; level++) {
        mg_relax(m, level, m->prm.nu1, ORC_RO_RED_BLACK);
        mg_clear_zero(m, level + 1);
        mg_apply_bc(m, level + 1);
        if (level == 0) {
          double residual;
          mg_restrict_residuals(m, 0, 1, (conv & OCU_CONVERGENCE_CALC_L2) ? rl2 : 0,
                                (conv & OCU_CONVERGENCE_CALC_LINF) ? rlinf : 0);
          residual = mg_pick(conv, *rl2, *rlinf);
          if (residual < tolerance) {
            mg_apply_bc(m, 0);
            m->last_vcycles = num_vcyc;
            return 1;
          }
        } else {
          mg_restrict_residuals(m, level, level + 1, 0, 0);
        }
      }
      mg_relax(m, coarse_level, mg_coarse_iters(m),
               m->prm.make_symmetric_operator ? ORC_RO_SYMMETRIC : ORC_RO_RED_BLACK);
      for (level = coarse_level - 1; level >= fine_level; level--) {
        mg_prolong(m, level + 1, level);
        if (level > 0)
          mg_relax(m, level, m->prm.nu2,
                   m->prm.make_symmetric_operator ? ORC_RO_BLACK_RED : ORC_RO_RED_BLACK);
      }
    }
    if (fine_level > 0) mg_prolong(m, fine_level, fine_level - 1);
  }
  m->last_vcycles = num_vcyc;
  return 0;
}

/* do_vcycle (sol_mgpressure3d.cpp:253-329) */
static int mg_do_vcycle(orc_mg *m, double tolerance, int max_iter, double *rl2, double *rlinf)
{
  const int conv = m->prm.convergence;
  const int coarse_level = m->num_levels - 1;
  int level, i_cyc;
  double orig_l2 = 0, orig_linf = 0, orig_error;
  mg_apply_bc(m, 0);
  mg_restrict_residuals(m, 0, 0, (conv & OCU_CONVERGENCE_CALC_L2) ? &orig_l2 : 0,
                        (conv & OCU_CONVERGENCE_CALC_LINF) ? &orig_linf : 0);
  orig_error = mg_pick(conv, orig_l2, orig_linf);
  if (orig_error < tolerance) {
    if (conv & OCU_CONVERGENCE_CALC_L2) *rl2 = orig_l2;
    if (conv & OCU_CONVERGENCE_CALC_LINF) *rlinf = orig_linf;
    return 1;
  }
  for (i_cyc = 0; i_cyc < max_iter; i_cyc++) {
    for (level = 0; level < coarse_level; level++) {
      mg_relax(m, level, m->prm.nu1, ORC_RO_RED_BLACK);
      mg_clear_zero(m, level + 1);
      mg_apply_bc(m, level + 1);
      if (level == 0) {
        double residual;
        mg_restrict_residuals(m, 0, 1, (conv & OCU_CONVERGENCE_CALC_L2) ? rl2 : 0,
                              (conv & OCU_CONVERGENCE_CALC_LINF) ? rlinf : 0);
        residual = mg_pick(conv, *rl2, *rlinf);
        if (residual < tolerance) {
          mg_apply_bc(m, 0);
          return 1;
        }
      } else {
        mg_restrict_residuals(m, level, level + 1, 0, 0);
      }
    }
    mg_relax(m, coarse_level, mg_coarse_iters(m),
             m->prm.make_symmetric_operator ? ORC_RO_SYMMETRIC : ORC_RO_RED_BLACK);
    for (level = coarse_level - 1; level >= 0; level--) {
      mg_prolong(m, level + 1, level);
      if (level > 0)
        mg_relax(m, level, m->prm.nu2,
                 m->prm.make_symmetric_operator ? ORC_RO_BLACK_RED : ORC_RO_RED_BLACK);
    }
  }
  return 0;
}

/* Sol_MultigridPressureMixed3DDeviceD::do_fmg (sol_mgpressuremixed3ddevd.cpp:79-100) */
static int mgmixed_do_fmg(orc_mg *m, double tolerance, int max_iter, double *rl2, double *rlinf)
{
  const ocu_layout *L = &m->cd->lay[0];
  long long n;
  for (n = 0; n < L->allocated; n++) m->rhs_f[n] = (float)m->cd->b[0][n];
  m->double_mode = 0;
  mg_do_fmg(m, tolerance > 1e-2 ? tolerance : 1e-2, 4, rl2, rlinf);
  for (n = 0; n < L->allocated; n++) m->cd->u[0][n] = (double)m->cf->u[0][n];
  m->double_mode = 1;
  if (tolerance < 1e-2 || m->prm.convergence == OCU_CONVERGENCE_L2) {
    int ok = mg_do_fmg(m, tolerance, max_iter, rl2, rlinf);
    for (n = 0; n < L->allocated; n++) m->cf->u[0][n] = (float)m->cd->u[0][n];
    return ok;
  }
  return 1;
}

#define IDXL(L, i, j, k) ((L)->shift + (long long)(i) * (L)->xstride + (long long)(j) * (L)->ystride + (long long)(k))

/* FP64 residual of the outer iteration + its norms (RMS via the reference reduction tree in
 * double). */
static void ir_residual(orc_mg *m, double *l2, double *linf)
{
  core_restrict_residuals_d(m->cd, 0, 0, l2, linf);
}

/* FP32-in-FP64 iterative refinement (no reference counterpart): x64 <- x64 + FP32 FMG
 * correction of A e = (float)(b - A x64), residual and norms in FP64. */
static int mgir_solve(orc_mg *m, double tolerance, int max_outer, double *rl2, double *rlinf)
{
  const int conv = m->prm.convergence;
  const ocu_layout *L = &m->cd->lay[0];
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  double l2 = 0, linf = 0, el2, elinf;
  int outer, i, j, k;
  orc_mg inner = *m;
  inner.kind = ORC_KIND_F;
  inner.double_mode = 0;
  inner.prm.convergence = OCU_CONVERGENCE_NONE;
  m->outer_iters = 0;
  m->double_mode = 1;
  core_apply_bc_d(m->cd, 0);
  ir_residual(m, &l2, &linf);
  *rl2 = l2; *rlinf = linf;
  if (mg_pick(conv, l2, linf) < tolerance) return 1;
  for (outer = 1; outer <= max_outer; outer++) {
    const double *r = m->cd->r[0];
    float *bf = m->cf->b[0];
    float *e;
    double *x = m->cd->u[0];
    for (i = 0; i < nx; i++)
      for (j = 0; j < ny; j++)
        for (k = 0; k < nz; k++) bf[IDXL(L, i, j, k)] = (float)r[IDXL(L, i, j, k)];
    core_clear_zero_f(m->cf, 0);
    mg_do_fmg(&inner, 0.0, m->inner_cycles - 1, &el2, &elinf);
    e = m->cf->u[0];
    for (i = 0; i < nx; i++)
      for (j = 0; j < ny; j++)
        for (k = 0; k < nz; k++) x[IDXL(L, i, j, k)] = x[IDXL(L, i, j, k)] + (double)e[IDXL(L, i, j, k)];
    core_apply_bc_d(m->cd, 0);
    ir_residual(m, &l2, &linf);
    m->outer_iters = outer;
    *rl2 = l2; *rlinf = linf;
    if (mg_pick(conv, l2, linf) < tolerance) return 1;
  }
  return 0;
}

static orc_mg *mg_alloc(int kind, const orc_mg_params *prm)
{
  orc_mg *m = (orc_mg *)calloc(1, sizeof(orc_mg));
  m->kind = kind;
  m->prm = *prm;
  return m;
}

orc_mg *orc_mg_create(int dtype, const orc_mg_params *prm, int nx, int ny, int nz, double hx,
                      double hy, double hz, void *rhs, const ocu_layout *rl)
{
  orc_mg *m;
  if (rl->gx < 1 || rl->gy < 1 || rl->gz < 1) return 0;
  m = mg_alloc(dtype == OCU_F64 ? ORC_KIND_D : ORC_KIND_F, prm);
  if (dtype == OCU_F64) {
    m->cd = core_create_d(&prm->bc, prm->disable_relax_on_host, nx, ny, nz, hx, hy, hz, (double *)rhs, rl);
    m->num_levels = m->cd->num_levels; m->dim = m->cd->dim; m->double_mode = 1;
  } else {
    m->cf = core_create_f(&prm->bc, prm->disable_relax_on_host, nx, ny, nz, hx, hy, hz, (float *)rhs, rl);
    m->num_levels = m->cf->num_levels; m->dim = m->cf->dim; m->double_mode = 0;
  }
  return m;
}

orc_mg *orc_mgmixed_create(const orc_mg_params *prm, int nx, int ny, int nz, double hx,
                           double hy, double hz, double *rhs, const ocu_layout *rl)
{
  orc_mg *m = mg_alloc(ORC_KIND_MIXED, prm);
  m->cd = core_create_d(&prm->bc, prm->disable_relax_on_host, nx, ny, nz, hx, hy, hz, rhs, rl);
  m->rhs_f = (float *)calloc(rl->allocated, sizeof(float));
  m->cf = core_create_f(&prm->bc, prm->disable_relax_on_host, nx, ny, nz, hx, hy, hz, m->rhs_f, rl);
  m->num_levels = m->cd->num_levels; m->dim = m->cd->dim;
  return m;
}

orc_mg *orc_mgir_create(const orc_mg_params *prm, int nx, int ny, int nz, double hx, double hy,
                        double hz, double *rhs, const ocu_layout *rl, int inner_cycles)
{
  orc_mg *m = mg_alloc(ORC_KIND_IR, prm);
  ocu_bc_set hom = prm->bc;
  orc_make_homogeneous(&hom);
  m->cd = core_create_d(&prm->bc, prm->disable_relax_on_host, nx, ny, nz, hx, hy, hz, rhs, rl);
  m->rhs_f = (float *)calloc(rl->allocated, sizeof(float));
  m->cf = core_create_f(&hom, prm->disable_relax_on_host, nx, ny, nz, hx, hy, hz, m->rhs_f, rl);
  m->num_levels = m->cd->num_levels; m->dim = m->cd->dim;
  m->inner_cycles = inner_cycles < 1 ? 1 : inner_cycles;
  m->double_mode = 1;
  return m;
}

void orc_mg_destroy(orc_mg *m)
{
  if (!m) return;
  core_destroy_f(m->cf);
  core_destroy_d(m->cd);
  free(m->rhs_f);
  free(m);
}

void orc_mg_set_params(orc_mg *m, const orc_mg_params *prm)
{
  m->prm = *prm;
  if (m->cf) { m->cf->bc = prm->bc; m->cf->disable_relax_on_host = prm->disable_relax_on_host; }
  if (m->cd) { m->cd->bc = prm->bc; m->cd->disable_relax_on_host = prm->disable_relax_on_host; }
  if (m->kind == ORC_KIND_IR && m->cf) orc_make_homogeneous(&m->cf->bc);
}

static int mg_fmg_dispatch(orc_mg *m, double tol, int max_iter, double *l2, double *linf)
{
  if (m->kind == ORC_KIND_MIXED) return mgmixed_do_fmg(m, tol, max_iter, l2, linf);
  if (m->kind == ORC_KIND_IR) return mgir_solve(m, tol, max_iter, l2, linf);
  return mg_do_fmg(m, tol, max_iter, l2, linf);
}

/* Base::solve (sol_mgpressure3d.cpp:332-370) */
int orc_mg_solve(orc_mg *m, double *residual, double tolerance, int max_iter)
{
  double l2 = 0, linf = 0;
  if (!orc_check_float((float)tolerance) || tolerance < 0 || max_iter <= 0) return 0;
  if (!mg_fmg_dispatch(m, tolerance, max_iter, &l2, &linf)) {
    mg_clear_zero(m, 0);
    if (!mg_fmg_dispatch(m, tolerance, max_iter, &l2, &linf)) {
      *residual = (m->prm.convergence == OCU_CONVERGENCE_L2) ? l2 : linf;
      return 0;
    }
  }
  *residual = (m->prm.convergence == OCU_CONVERGENCE_L2) ? l2 : linf;
  return 1;
}

int orc_mg_run_vcycles(orc_mg *m, int count)
{
  double l2, linf;
  if (count <= 0) return 0;
  mg_do_vcycle(m, 0, count, &l2, &linf);
  return 1;
}

int orc_mg_run_fmg(orc_mg *m, int count)
{
  double l2, linf;
  if (count < 0) return 0;
  mg_do_fmg(m, 0, count, &l2, &linf);
  return 1;
}

/* Level operations on one hierarchy (core 0 = interface precision, 1 = FP32 hierarchy). */
static int core_is_f(const orc_mg *m, int core) { return core == 1 || m->kind == ORC_KIND_F; }

int orc_mg_relax(orc_mg *m, int core, int level, int iterations, int order)
{
  if (core_is_f(m, core)) core_relax_f(m->cf, level, iterations, order);
  else core_relax_d(m->cd, level, iterations, order);
  return 1;
}

int orc_mg_relax_sweep(orc_mg *m, int core, int level, int color)
{
  if (core_is_f(m, core)) core_relax_color_f(m->cf, level, color & 1);
  else core_relax_color_d(m->cd, level, color & 1);
  return 1;
}

int orc_mg_restrict_residuals(orc_mg *m, int core, int fine, int coarse, double *l2, double *linf)
{
  if (core_is_f(m, core)) core_restrict_residuals_f(m->cf, fine, coarse, l2, linf);
  else core_restrict_residuals_d(m->cd, fine, coarse, l2, linf);
  return 1;
}

int orc_mg_prolong(orc_mg *m, int core, int coarse, int fine)
{
  if (core_is_f(m, core)) core_prolong_bc_f(m->cf, coarse, fine);
  else core_prolong_bc_d(m->cd, coarse, fine);
  return 1;
}

int orc_mg_num_levels(const orc_mg *m) { return m->num_levels; }
int orc_mg_vcycles(const orc_mg *m) { return m->last_vcycles; }
int orc_mgir_outer_iterations(const orc_mg *m) { return m->outer_iters; }
double orc_mg_omega(const orc_mg *m) { return m->cd ? m->cd->omega : m->cf->omega; }

void *orc_mg_grid(orc_mg *m, char which, int level, ocu_layout *lo)
{
  int use_d = (m->kind == ORC_KIND_D || m->kind == ORC_KIND_MIXED || m->kind == ORC_KIND_IR);
  if (which == 'U' || which == 'B' || which == 'R') { use_d = 0; which = (char)(which - 'A' + 'a'); }
  if (use_d) {
    if (lo) *lo = m->cd->lay[level];
    return which == 'u' ? (void *)m->cd->u[level] : which == 'b' ? (void *)m->cd->b[level] : (void *)m->cd->r[level];
  }
  if (lo) *lo = m->cf->lay[level];
  return which == 'u' ? (void *)m->cf->u[level] : which == 'b' ? (void *)m->cf->b[level] : (void *)m->cf->r[level];
}

/* ------------------------------------------------------------------------------------------
 * Projection (sol_project3d.cpp:26-68, sol_project3ddev.cu:28-135)
 * ---------------------------------------------------------------------------------------- */
struct orc_project {
  int dtype;
  ocu_bc_set bc;
  int nx, ny, nz;
  double hx, hy, hz;
  void *u, *v, *w;
  ocu_layout L;    /* shared MAC layout (strides/shift) */
  ocu_layout Ldiv; /* divergence: interior (nx,ny,nz), same padded extents */
  void *div;
  orc_mg *mg;
};

static ocu_bc orc_convert_bc(const ocu_bc *b)
{
  ocu_bc r;
  r.type = OCU_BC_INVALID; r.value = 0; r.aux_value = 0;
  if (b->type == OCU_BC_PERIODIC) r.type = OCU_BC_PERIODIC;
  else if (b->type == OCU_BC_FORCED_INFLOW_VARIABLE_SLIP) { r.type = OCU_BC_NEUMANN; r.value = 0; }
  return r;
}

/* kind: 0 = Sol_ProjectDivergence3DDevice<float>, 1 = <double>, 2 =
 * Sol_ProjectDivergenceMixed3DDeviceD (the reference mixed pressure solver,
 * sol_projectmixed3d.cu:48-91), 3 = the same with the FP32-in-FP64 refinement solver. */
orc_project *orc_project_create_kind(int kind, const ocu_bc_set *bc, int nx, int ny, int nz,
                                     double hx, double hy, double hz, void *u, void *v, void *w,
                                     const ocu_layout *Lm, int inner_cycles)
{
  orc_project *p = (orc_project *)calloc(1, sizeof(orc_project));
  orc_mg_params prm;
  const int dtype = kind == 0 ? OCU_F32 : OCU_F64;
  size_t es = dtype == OCU_F64 ? 8 : 4;
  p->dtype = dtype; p->bc = *bc;
  p->nx = nx; p->ny = ny; p->nz = nz; p->hx = hx; p->hy = hy; p->hz = hz;
  p->u = u; p->v = v; p->w = w; p->L = *Lm;
  orc_layout(nx, ny, nz, 1, 1, 1, Lm->pnx - (nx + 2), Lm->pny - (ny + 2), Lm->pnz - (nz + 2), &p->Ldiv);
  p->div = calloc(p->Ldiv.allocated, es);
  memset(&prm, 0, sizeof(prm));
  prm.bc.xneg = orc_convert_bc(&bc->xneg); prm.bc.xpos = orc_convert_bc(&bc->xpos);
  prm.bc.yneg = orc_convert_bc(&bc->yneg); prm.bc.ypos = orc_convert_bc(&bc->ypos);
  prm.bc.zneg = orc_convert_bc(&bc->zneg); prm.bc.zpos = orc_convert_bc(&bc->zpos);
  prm.nu1 = 2; prm.nu2 = 2;
  prm.convergence = OCU_CONVERGENCE_LINF;
  if (kind == 2)
    p->mg = orc_mgmixed_create(&prm, nx, ny, nz, hx, hy, hz, (double *)p->div, &p->Ldiv);
  else if (kind == 3)
    p->mg = orc_mgir_create(&prm, nx, ny, nz, hx, hy, hz, (double *)p->div, &p->Ldiv, inner_cycles);
  else
    p->mg = orc_mg_create(dtype, &prm, nx, ny, nz, hx, hy, hz, p->div, &p->Ldiv);
  return p;
}

orc_project *orc_project_create(int dtype, const ocu_bc_set *bc, int nx, int ny, int nz,
                                double hx, double hy, double hz, void *u, void *v, void *w,
                                const ocu_layout *Lm)
{
  return orc_project_create_kind(dtype == OCU_F64 ? 1 : 0, bc, nx, ny, nz, hx, hy, hz, u, v, w, Lm, 4);
}

void orc_project_destroy(orc_project *p)
{
  if (!p) return;
  orc_mg_destroy(p->mg);
  free(p->div);
  free(p);
}

int orc_project_solve_divergence_only(orc_project *p)
{
  int ok = 1;
  if (p->dtype == OCU_F64) {
    ok &= orc_mac_bc_level1_d((double *)p->u, (double *)p->v, (double *)p->w, &p->L, p->nx, p->ny, p->nz, &p->bc, p->hx, p->hy, p->hz);
    orc_divergence_d((double *)p->u, (double *)p->v, (double *)p->w, (double *)p->div, &p->L, p->nx, p->ny, p->nz, p->hx, p->hy, p->hz);
  } else {
    ok &= orc_mac_bc_level1_f((float *)p->u, (float *)p->v, (float *)p->w, &p->L, p->nx, p->ny, p->nz, &p->bc, p->hx, p->hy, p->hz);
    orc_divergence_f((float *)p->u, (float *)p->v, (float *)p->w, (float *)p->div, &p->L, p->nx, p->ny, p->nz, p->hx, p->hy, p->hz);
  }
  return ok;
}

int orc_project_solve(orc_project *p, double tolerance)
{
  double residual = 0;
  int ok = orc_project_solve_divergence_only(p);
  ok &= orc_mg_solve(p->mg, &residual, tolerance, 15);
  if (p->dtype == OCU_F64) {
    orc_gradient_d((double *)p->u, (double *)p->v, (double *)p->w, p->mg->cd->u[0], &p->L, p->nx, p->ny, p->nz, p->hx, p->hy, p->hz, -1);
    ok &= orc_mac_bc_level1_d((double *)p->u, (double *)p->v, (double *)p->w, &p->L, p->nx, p->ny, p->nz, &p->bc, p->hx, p->hy, p->hz);
  } else {
    orc_gradient_f((float *)p->u, (float *)p->v, (float *)p->w, p->mg->cf->u[0], &p->L, p->nx, p->ny, p->nz, p->hx, p->hy, p->hz, -1);
    ok &= orc_mac_bc_level1_f((float *)p->u, (float *)p->v, (float *)p->w, &p->L, p->nx, p->ny, p->nz, &p->bc, p->hx, p->hy, p->hz);
  }
  return ok;
}

void *orc_project_divergence(orc_project *p) { return p->div; }
orc_mg *orc_project_pressure_solver(orc_project *p) { return p->mg; }

/* ------------------------------------------------------------------------------------------
 * Sol_PCGPressure3DDevice<T> (ocuequation/sol_pcgpressure3d.cu:289-654).
 * ---------------------------------------------------------------------------------------- */
struct orc_pcg {
  int dtype;
  orc_pcg_params prm;
  int nx, ny, nz;
  double h, fx, fy, fz;
  ocu_layout L;
  void *rhs, *coef;          /* borrowed */
  void *p, *r, *y, *d;       /* pressure, residual (the multigrid's rhs), L d, search direction */
  orc_mg *mg;
  int iterations;
};

orc_pcg *orc_pcg_create(int dtype, const orc_pcg_params *prm, int nx, int ny, int nz, double hx_d, double hy_d,
                        double hz_d, void *rhs, void *coefficient, const ocu_layout *L)
{
  const float hx = (float)hx_d, hy = (float)hy_d, hz = (float)hz_d;
  const size_t es = dtype == OCU_F64 ? 8 : 4;
  orc_mg_params mp;
  orc_pcg *p;
  int f;
  const ocu_bc *faces[6];
  if (L->gx < 1 || L->gy < 1 || L->gz < 1) return 0;
  faces[0] = &prm->bc.xpos; faces[1] = &prm->bc.xneg; faces[2] = &prm->bc.ypos;
  faces[3] = &prm->bc.yneg; faces[4] = &prm->bc.zpos; faces[5] = &prm->bc.zneg;
  for (f = 0; f < 6; f++) /* bc.check_type(BC_PERIODIC, BC_NEUMANN) */
    if (faces[f]->type != OCU_BC_PERIODIC && faces[f]->type != OCU_BC_NEUMANN) return 0;
  p = (orc_pcg *)calloc(1, sizeof(orc_pcg));
  p->dtype = dtype;
  p->prm = *prm;
  p->nx = nx; p->ny = ny; p->nz = nz;
  p->h = orc_min3(hx, hy, hz);
  p->fx = (p->h * p->h) / ((double)hx * hx);
  p->fy = (p->h * p->h) / ((double)hy * hy);
  p->fz = (p->h * p->h) / ((double)hz * hz);
  p->L = *L;
  p->rhs = rhs;
  p->coef = coefficient;
  p->p = calloc((size_t)L->allocated, es);
  p->r = calloc((size_t)L->allocated, es);
  p->y = calloc((size_t)L->allocated, es);
  p->d = calloc((size_t)L->allocated, es);
  memset(&mp, 0, sizeof(mp));
  mp.bc = prm->bc;
  mp.nu1 = 2;
  mp.nu2 = 2;
  mp.convergence = OCU_CONVERGENCE_NONE_CALC_L2LINF;
  p->mg = orc_mg_create(dtype, &mp, nx, ny, nz, hx, hy, hz, p->r, L);
  return p;
}

void orc_pcg_destroy(orc_pcg *p)
{
  if (!p) return;
  orc_mg_destroy(p->mg);
  free(p->p); free(p->r); free(p->y); free(p->d);
  free(p);
}

void *orc_pcg_pressure(orc_pcg *p) { return p->p; }
int orc_pcg_iterations(const orc_pcg *p) { return p->iterations; }

/* f / h^2 as the reference's host code has them: rounded to T */
static double pcg_fh(const orc_pcg *p, double f)
{
  return p->dtype == OCU_F64 ? f / (p->h * p->h) : (double)(float)(f / (p->h * p->h));
}

static void pcg_bc(orc_pcg *p, void *g)
{
  const double hx = p->h / sqrt(p->fx), hy = p->h / sqrt(p->fy), hz = p->h / sqrt(p->fz);
  if (p->dtype == OCU_F64) orc_bc_nocorners_dev_d((double *)g, &p->L, &p->prm.bc, hx, hy, hz);
  else orc_bc_nocorners_dev_f((float *)g, &p->L, &p->prm.bc, hx, hy, hz);
}

/* invoke_kernel_apply_laplacian: src's face ghosts first, then the stencil */
static void pcg_apply_laplacian(orc_pcg *p, void *dst, void *src)
{
  const double fxh = pcg_fh(p, p->fx), fyh = pcg_fh(p, p->fy), fzh = pcg_fh(p, p->fz);
  pcg_bc(p, src);
  if (p->dtype == OCU_F64)
    orc_pcg_laplacian_d((double *)dst, (const double *)src, (const double *)p->coef, &p->L, fxh, fyh, fzh);
  else orc_pcg_laplacian_f((float *)dst, (const float *)src, (const float *)p->coef, &p->L, fxh, fyh, fzh);
}

static void pcg_diag(orc_pcg *p, void *dst, const void *src)
{
  const double fxh = pcg_fh(p, p->fx), fyh = pcg_fh(p, p->fy), fzh = pcg_fh(p, p->fz);
  if (p->dtype == OCU_F64)
    orc_pcg_diag_d((double *)dst, (const double *)src, (const double *)p->coef, &p->L, fxh, fyh, fzh);
  else orc_pcg_diag_f((float *)dst, (const float *)src, (const float *)p->coef, &p->L, fxh, fyh, fzh);
}

static double pcg_dot(orc_pcg *p, const void *a, const void *b)
{
  return p->dtype == OCU_F64 ? orc_pcg_dot_d((const double *)a, (const double *)b, &p->L)
                             : orc_pcg_dot_f((const float *)a, (const float *)b, &p->L);
}

static void pcg_lincomb2(orc_pcg *p, void *res, double a1, const void *g1, double a2, const void *g2)
{
  if (p->dtype == OCU_F64) orc_lincomb2_d((double *)res, &p->L, a1, (const double *)g1, a2, (const double *)g2);
  else orc_lincomb2_f((float *)res, &p->L, a1, (const float *)g1, a2, (const float *)g2);
}

/* apply_preconditioner (sol_pcgpressure3d.cu:289-331); the multigrid solves for its own rhs,
 * the residual grid, whatever src is */
static void pcg_precondition(orc_pcg *p, void *dst, const void *src)
{
  const int pc = p->prm.preconditioner;
  const size_t es = p->dtype == OCU_F64 ? 8 : 4;
  if (pc == OCU_PRECOND_JACOBI) {
    pcg_diag(p, dst, src);
  } else if (pc == OCU_PRECOND_MULTIGRID || pc == OCU_PRECOND_BFBT) {
    void *u = orc_mg_grid(p->mg, 'u', 0, 0);
    memset(u, 0, es * (size_t)p->L.allocated);
    if (p->prm.multigrid_use_fmg) orc_mg_run_fmg(p->mg, p->prm.multigrid_cycles);
    else orc_mg_run_vcycles(p->mg, p->prm.multigrid_cycles);
    if (p->dtype == OCU_F64) orc_lincomb1_d((double *)dst, &p->L, -1.0, (const double *)u);
    else orc_lincomb1_f((float *)dst, &p->L, -1.0, (const float *)u);
    if (pc == OCU_PRECOND_BFBT) pcg_diag(p, dst, dst);
  } else {
    memcpy(dst, src, es * (size_t)p->L.allocated);
  }
}

/* the host scalars of do_pcg are T */
static double pcg_round(const orc_pcg *p, double x) { return p->dtype == OCU_F64 ? x : (double)(float)x; }

/* do_pcg (sol_pcgpressure3d.cu:335-457) and solve (:571-601) */
int orc_pcg_solve(orc_pcg *p, double *residual, double tolerance, int max_iter)
{
  double delta0, deltanew, deltaold, d_dot_y, alpha, beta, l2, linf;
  int it = 0, converged, ok;
  if (!orc_check_float((float)tolerance) || tolerance < 0 || max_iter <= 0) return 0;
  pcg_bc(p, p->coef);
  pcg_apply_laplacian(p, p->y, p->p);
  pcg_lincomb2(p, p->r, 1.0, p->rhs, -1.0, p->y);
  pcg_precondition(p, p->d, p->r);
  delta0 = pcg_dot(p, p->r, p->d);
  deltanew = delta0;
  converged = (it > max_iter) || (delta0 < tolerance * tolerance);
  while (!converged) {
    pcg_apply_laplacian(p, p->y, p->d);
    d_dot_y = pcg_dot(p, p->d, p->y);
    alpha = pcg_round(p, deltanew / d_dot_y);
    pcg_lincomb2(p, p->p, 1.0, p->p, alpha, p->d);
    if (it % 25 == 0) {
      pcg_apply_laplacian(p, p->y, p->p);
      pcg_lincomb2(p, p->r, 1.0, p->rhs, -1.0, p->y);
    } else {
      pcg_lincomb2(p, p->r, 1.0, p->r, -alpha, p->y);
    }
    pcg_precondition(p, p->y, p->r);
    deltaold = deltanew;
    deltanew = pcg_dot(p, p->r, p->y);
    beta = pcg_round(p, deltanew / deltaold);
    pcg_lincomb2(p, p->d, beta, p->d, 1.0, p->y);
    it++;
    converged = (it > max_iter) || (deltanew < tolerance * tolerance);
  }
  ok = deltanew <= tolerance * tolerance;
  p->iterations = it;
  l2 = sqrt(deltanew);
  linf = p->dtype == OCU_F64 ? orc_reduce_d((const double *)p->r, &p->L, OCU_REDUCE_MAXABS)
                             : orc_reduce_f((const float *)p->r, &p->L, OCU_REDUCE_MAXABS);
  *residual = p->prm.convergence == OCU_CONVERGENCE_L2 ? l2 : linf;
  return ok;
}

/* ------------------------------------------------------------------------------------------
 * Eqn_IncompressibleNS3D<T> (eqn_incompressns3d.cu:164-399) and Equation::advance
 * (equation.cpp:31-56).  Parameters that the reference stores as T are rounded to T here.
 * ---------------------------------------------------------------------------------------- */
struct orc_ns {
  int dtype;
  orc_ns_params prm;
  double T_gravity, T_bouyancy, T_kappa, T_nu; /* values after rounding to T */
  ocu_layout Lu, Lv, Lw, Lt;
  void *u, *v, *w, *t, *du, *dv, *dw, *dt, *ldu, *ldv, *ldw, *ldt;
  double lastdt;
  int num_steps;
  orc_project *proj;
};

static double rt(int dtype, double x) { return dtype == OCU_F64 ? x : (double)(float)x; }

void orc_ns_set_omp_threads(int n)
{
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

orc_ns *orc_ns_create(int dtype, const orc_ns_params *prm, const void *iu, const void *iv,
                      const void *iw, const void *it)
{
  orc_ns *ns = (orc_ns *)calloc(1, sizeof(orc_ns));
  size_t es = dtype == OCU_F64 ? 8 : 4;
  const int nx = prm->nx, ny = prm->ny, nz = prm->nz;
  ns->dtype = dtype;
  ns->prm = *prm;
  ns->T_gravity = rt(dtype, prm->gravity);
  ns->T_bouyancy = rt(dtype, prm->bouyancy);
  ns->T_kappa = rt(dtype, prm->thermal_diffusion);
  ns->T_nu = rt(dtype, prm->viscosity);
  orc_layout(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1, &ns->Lu);
  orc_layout(nx, ny + 1, nz, 1, 1, 1, 1, 0, 1, &ns->Lv);
  orc_layout(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0, &ns->Lw);
  orc_layout(nx, ny, nz, 1, 1, 1, 1, 1, 1, &ns->Lt);
#define NSALLOC(p, L) p = calloc((L).allocated, es)
  NSALLOC(ns->u, ns->Lu); NSALLOC(ns->du, ns->Lu); NSALLOC(ns->ldu, ns->Lu);
  NSALLOC(ns->v, ns->Lv); NSALLOC(ns->dv, ns->Lv); NSALLOC(ns->ldv, ns->Lv);
  NSALLOC(ns->w, ns->Lw); NSALLOC(ns->dw, ns->Lw); NSALLOC(ns->ldw, ns->Lw);
  NSALLOC(ns->t, ns->Lt); NSALLOC(ns->dt, ns->Lt); NSALLOC(ns->ldt, ns->Lt);
#undef NSALLOC
  memcpy(ns->u, iu, es * ns->Lu.allocated);
  memcpy(ns->v, iv, es * ns->Lv.allocated);
  memcpy(ns->w, iw, es * ns->Lw.allocated);
  memcpy(ns->t, it, es * ns->Lt.allocated);
  ns->proj = orc_project_create(dtype, &prm->flow_bc, nx, ny, nz, prm->hx, prm->hy, prm->hz, ns->u, ns->v, ns->w, &ns->Lu);
  if (dtype == OCU_F64) {
    orc_mac_bc_level1_d((double *)ns->u, (double *)ns->v, (double *)ns->w, &ns->Lu, nx, ny, nz, &prm->flow_bc, prm->hx, prm->hy, prm->hz);
    orc_bc_level1_d((double *)ns->t, &ns->Lt, &prm->temp_bc, prm->hx, prm->hy, prm->hz);
  } else {
    orc_mac_bc_level1_f((float *)ns->u, (float *)ns->v, (float *)ns->w, &ns->Lu, nx, ny, nz, &prm->flow_bc, prm->hx, prm->hy, prm->hz);
    orc_bc_level1_f((float *)ns->t, &ns->Lt, &prm->temp_bc, prm->hx, prm->hy, prm->hz);
  }
  return ns;
}

void orc_ns_destroy(orc_ns *ns)
{
  if (!ns) return;
  orc_project_destroy(ns->proj);
  free(ns->u); free(ns->v); free(ns->w); free(ns->t);
  free(ns->du); free(ns->dv); free(ns->dw); free(ns->dt);
  free(ns->ldu); free(ns->ldv); free(ns->ldw); free(ns->ldt);
  free(ns);
}

/* get_max_stable_timestep (eqn_incompressns3d.cu:301-328) */
double orc_ns_get_max_stable_timestep(orc_ns *ns)
{
  const orc_ns_params *p = &ns->prm;
  double mu, mv, mw, ut, vt, wt, step, minh;
  if (ns->dtype == OCU_F64) {
    mu = orc_reduce_d((double *)ns->u, &ns->Lu, OCU_REDUCE_MAXABS);
    mv = orc_reduce_d((double *)ns->v, &ns->Lv, OCU_REDUCE_MAXABS);
    mw = orc_reduce_d((double *)ns->w, &ns->Lw, OCU_REDUCE_MAXABS);
  } else {
    mu = orc_reduce_f((float *)ns->u, &ns->Lu, OCU_REDUCE_MAXABS);
    mv = orc_reduce_f((float *)ns->v, &ns->Lv, OCU_REDUCE_MAXABS);
    mw = orc_reduce_f((float *)ns->w, &ns->Lw, OCU_REDUCE_MAXABS);
  }
  ut = p->hx / mu; vt = p->hy / mv; wt = p->hz / mw;
  if (!orc_check_float((float)ut)) ut = 1e10;
  if (!orc_check_float((float)vt)) vt = 1e10;
  if (!orc_check_float((float)wt)) wt = 1e10;
  step = p->cfl_factor * orc_min3(ut, vt, wt);
  minh = orc_min3(p->hx, p->hy, p->hz);
  if (ns->T_kappa > 0) {
    double d = rt(ns->dtype, 6 * ns->T_kappa);
    double c = (minh * minh) / d;
    step = step < c ? step : c;
  }
  if (ns->T_nu > 0) {
    double d = rt(ns->dtype, 6 * ns->T_nu);
    double c = (minh * minh) / d;
    step = step < c ? step : c;
  }
  return step;
}

/* advance_one_step (eqn_incompressns3d.cu:331-399) */
int orc_ns_advance_one_step(orc_ns *ns, double dtv)
{
  const orc_ns_params *p = &ns->prm;
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const int vd = p->vertical_direction;
  int ok = 1;
  double dm = (vd & OCU_DIR_NEGATIVE_FLAG) ? 1 : -1;
  double coef = rt(ns->dtype, rt(ns->dtype, dm * ns->T_gravity) * ns->T_bouyancy);
  int nbr = (vd & OCU_DIR_XAXIS_FLAG) ? ns->Lt.xstride : (vd & OCU_DIR_YAXIS_FLAG) ? ns->Lt.ystride : 1;
  double ab = rt(ns->dtype, -dtv * dtv / (2 * ns->lastdt));
  int ab2 = (p->time_step == OCU_TS_ADAMS_BASHFORD2 && ns->lastdt > 0);
  ns->num_steps++;
  if (ns->dtype == OCU_F64) {
    double *u = (double *)ns->u, *v = (double *)ns->v, *w = (double *)ns->w, *t = (double *)ns->t;
    double *du = (double *)ns->du, *dv = (double *)ns->dv, *dw = (double *)ns->dw, *dT = (double *)ns->dt;
    double *vert = (vd & OCU_DIR_XAXIS_FLAG) ? du : (vd & OCU_DIR_YAXIS_FLAG) ? dv : dw;
    orc_advect_self_d(u, v, w, du, dv, dw, &ns->Lu, nx, ny, nz, p->hx, p->hy, p->hz, p->advection_scheme);
    if (ns->T_nu > 0) {
      orc_laplacian_d(u, du, &ns->Lu, nx + 1, ny, nz, p->hx, p->hy, p->hz, ns->T_nu);
      orc_laplacian_d(v, dv, &ns->Lu, nx, ny + 1, nz, p->hx, p->hy, p->hz, ns->T_nu);
      orc_laplacian_d(w, dw, &ns->Lu, nx, ny, nz + 1, p->hx, p->hy, p->hz, ns->T_nu);
    }
    orc_thermal_force_d(vert, coef, t, &ns->Lt, nbr, nx, ny, nz);
    orc_advect_passive_d(u, v, w, t, dT, &ns->Lt, nx, ny, nz, p->hx, p->hy, p->hz, p->advection_scheme);
    if (ns->T_kappa > 0) orc_laplacian_d(t, dT, &ns->Lt, nx, ny, nz, p->hx, p->hy, p->hz, ns->T_kappa);
    if (ab2) {
      orc_lincomb2_d(t, &ns->Lt, 1.0, t, rt(1, dtv - ab), dT);
      orc_lincomb2_d(t, &ns->Lt, 1.0, t, ab, (double *)ns->ldt);
    } else {
      orc_lincomb2_d(t, &ns->Lt, 1.0, t, dtv, dT);
    }
    ok &= orc_bc_nocorners_dev_d(t, &ns->Lt, &p->temp_bc, p->hx, p->hy, p->hz);
    if (ab2) {
      orc_lincomb2_d(u, &ns->Lu, 1.0, u, dtv - ab, du); orc_lincomb2_d(u, &ns->Lu, 1.0, u, ab, (double *)ns->ldu);
      orc_lincomb2_d(v, &ns->Lv, 1.0, v, dtv - ab, dv); orc_lincomb2_d(v, &ns->Lv, 1.0, v, ab, (double *)ns->ldv);
      orc_lincomb2_d(w, &ns->Lw, 1.0, w, dtv - ab, dw); orc_lincomb2_d(w, &ns->Lw, 1.0, w, ab, (double *)ns->ldw);
    } else {
      orc_lincomb2_d(u, &ns->Lu, 1.0, u, dtv, du);
      orc_lincomb2_d(v, &ns->Lv, 1.0, v, dtv, dv);
      orc_lincomb2_d(w, &ns->Lw, 1.0, w, dtv, dw);
    }
    if (p->time_step == OCU_TS_ADAMS_BASHFORD2) {
      ns->lastdt = dtv;
      memcpy(ns->ldt, dT, 8 * ns->Lt.allocated);
      memcpy(ns->ldu, du, 8 * ns->Lu.allocated);
      memcpy(ns->ldv, dv, 8 * ns->Lv.allocated);
      memcpy(ns->ldw, dw, 8 * ns->Lw.allocated);
    }
  } else {
    float *u = (float *)ns->u, *v = (float *)ns->v, *w = (float *)ns->w, *t = (float *)ns->t;
    float *du = (float *)ns->du, *dv = (float *)ns->dv, *dw = (float *)ns->dw, *dT = (float *)ns->dt;
    float *vert = (vd & OCU_DIR_XAXIS_FLAG) ? du : (vd & OCU_DIR_YAXIS_FLAG) ? dv : dw;
    orc_advect_self_f(u, v, w, du, dv, dw, &ns->Lu, nx, ny, nz, p->hx, p->hy, p->hz, p->advection_scheme);
    if (ns->T_nu > 0) {
      orc_laplacian_f(u, du, &ns->Lu, nx + 1, ny, nz, p->hx, p->hy, p->hz, ns->T_nu);
      orc_laplacian_f(v, dv, &ns->Lu, nx, ny + 1, nz, p->hx, p->hy, p->hz, ns->T_nu);
      orc_laplacian_f(w, dw, &ns->Lu, nx, ny, nz + 1, p->hx, p->hy, p->hz, ns->T_nu);
    }
    orc_thermal_force_f(vert, coef, t, &ns->Lt, nbr, nx, ny, nz);
    orc_advect_passive_f(u, v, w, t, dT, &ns->Lt, nx, ny, nz, p->hx, p->hy, p->hz, p->advection_scheme);
    if (ns->T_kappa > 0) orc_laplacian_f(t, dT, &ns->Lt, nx, ny, nz, p->hx, p->hy, p->hz, ns->T_kappa);
    if (ab2) {
      orc_lincomb2_f(t, &ns->Lt, 1.0, t, rt(0, dtv - ab), dT);
      orc_lincomb2_f(t, &ns->Lt, 1.0, t, ab, (float *)ns->ldt);
    } else {
      orc_lincomb2_f(t, &ns->Lt, 1.0, t, dtv, dT);
    }
    ok &= orc_bc_nocorners_dev_f(t, &ns->Lt, &p->temp_bc, p->hx, p->hy, p->hz);
    if (ab2) {
      orc_lincomb2_f(u, &ns->Lu, 1.0, u, dtv - ab, du); orc_lincomb2_f(u, &ns->Lu, 1.0, u, ab, (float *)ns->ldu);
      orc_lincomb2_f(v, &ns->Lv, 1.0, v, dtv - ab, dv); orc_lincomb2_f(v, &ns->Lv, 1.0, v, ab, (float *)ns->ldv);
      orc_lincomb2_f(w, &ns->Lw, 1.0, w, dtv - ab, dw); orc_lincomb2_f(w, &ns->Lw, 1.0, w, ab, (float *)ns->ldw);
    } else {
      orc_lincomb2_f(u, &ns->Lu, 1.0, u, dtv, du);
      orc_lincomb2_f(v, &ns->Lv, 1.0, v, dtv, dv);
      orc_lincomb2_f(w, &ns->Lw, 1.0, w, dtv, dw);
    }
    if (p->time_step == OCU_TS_ADAMS_BASHFORD2) {
      ns->lastdt = dtv;
      memcpy(ns->ldt, dT, 4 * ns->Lt.allocated);
      memcpy(ns->ldu, du, 4 * ns->Lu.allocated);
      memcpy(ns->ldv, dv, 4 * ns->Lv.allocated);
      memcpy(ns->ldw, dw, 4 * ns->Lw.allocated);
    }
  }
  ok &= orc_project_solve(ns->proj, p->max_divergence);
  return ok;
}

/* Equation::advance (equation.cpp:31-56) */
int orc_ns_advance(orc_ns *ns, double dtv)
{
  double dtleft = dtv;
  if (!orc_check_float((float)dtv)) return 0;
  while (dtleft > 0) {
    int subds = (int)ceil(dtleft / orc_ns_get_max_stable_timestep(ns));
    double subdt = dtleft / subds;
    if (!orc_ns_advance_one_step(ns, subdt)) return 0;
    dtleft -= subdt;
  }
  return 1;
}

void *orc_ns_grid(orc_ns *ns, char which)
{
  switch (which) {
    case 'u': return ns->u; case 'v': return ns->v; case 'w': return ns->w; case 't': return ns->t;
    case 'U': return ns->du; case 'V': return ns->dv; case 'W': return ns->dw; case 'T': return ns->dt;
    case 'p': return orc_mg_grid(ns->proj->mg, 'u', 0, 0);
    default: return 0;
  }
}

void orc_ns_layout(orc_ns *ns, ocu_layout *out) { *out = ns->Lu; }
