/*
 * ref_driver.cu -- TEST INFRASTRUCTURE ONLY.
 *
 * A C entry layer over OpenCurrent's own device classes, compiled from the reference sources
 * by oracle/build_ref.sh into oracle/_ref/libocu_ref.so.  The GPU parity tests load it with
 * ctypes (oracle/ref_ctypes.py) to run the reference's solver on the same inputs as the
 * B200 library.  The product never links it.
 *
 * Every function only moves data in and out of the reference's Grid3DDevice / Grid3DHost
 * objects and calls the reference's public methods:
 *   Sol_MultigridPressure3DDevice<T>          ocuequation/sol_mgpressure3d.h:86-179
 *   Sol_MultigridPressureMixed3DDeviceD        ocuequation/sol_mgpressuremixed3d.h:28-55
 *   Sol_ProjectDivergence3DDevice<T>           ocuequation/sol_project3d.h:74-93
 *   Sol_ProjectDivergenceMixed3DDeviceD        ocuequation/sol_projectmixed3d.h:28-45
 *   Sol_SelfAdvection3DDevice<T>               ocuequation/sol_selfadvection3d.h:30-70
 *   Sol_PassiveAdvection3DDevice<T>            ocuequation/sol_passiveadvection3d.h:28-60
 *   Eqn_IncompressibleNS3D<T>                  ocuequation/eqn_incompressns3d.h:30-180
 * Plain-C parameter blocks are those of the CPU oracle (oracle/ocu_oracle.h), whose fields
 * are the reference's public fields one for one.
 */
#include <cstdio>
#include <cstring>

#include "ocuequation/eqn_incompressns3d.h"
#include "ocuequation/sol_mgpressure3d.h"
#include "ocuequation/sol_mgpressuremixed3d.h"
#include "ocuequation/sol_passiveadvection3d.h"
#include "ocuequation/sol_pcgpressure3d.h"
#include "ocuequation/sol_project3d.h"
#include "ocuequation/sol_projectmixed3d.h"
#include "ocuequation/sol_selfadvection3d.h"
#include "ocuutil/thread.h"

#include "../ocu_oracle.h"

using namespace ocu;

namespace {

bool g_ready = false;

bool ready() {
  if (!g_ready) {
    g_ready = ThreadManager::initialize(1) && ThreadManager::initialize_image(0);
  }
  return g_ready;
}

BoundaryCondition to_bc(const ocu_bc &b) {
  BoundaryCondition r;
  r.type = (BoundaryConditionType)b.type;
  r.value = b.value;
  r.aux_value = b.aux_value;
  return r;
}

BoundaryConditionSet to_bcset(const ocu_bc_set &s) {
  return BoundaryConditionSet(to_bc(s.xpos), to_bc(s.xneg), to_bc(s.ypos), to_bc(s.yneg),
                              to_bc(s.zpos), to_bc(s.zneg));
}

void fill_layout(const Grid3DUntyped &g, ocu_layout *L) {
  L->nx = g.nx();
  L->ny = g.ny();
  L->nz = g.nz();
  L->gx = g.gx();
  L->gy = g.gy();
  L->gz = g.gz();
  L->pnx = g.pnx();
  L->pny = g.pny();
  L->pnz = g.pnz();
  L->xstride = g.xstride();
  L->ystride = g.ystride();
  L->shift = g.shift_amount();
  L->allocated = g.num_allocated_elements();
}

/* A device grid of either precision; `borrowed` grids belong to a reference object. */
struct RefGrid {
  int dtype;
  Grid3DDevice<float> *f;
  Grid3DDevice<double> *d;
  bool borrowed;
  const Grid3DUntyped &untyped() const {
    return dtype == OCU_F64 ? (const Grid3DUntyped &)*d : (const Grid3DUntyped &)*f;
  }
  void *buffer() { return dtype == OCU_F64 ? (void *)d->buffer() : (void *)f->buffer(); }
  size_t bytes() const {
    return (size_t)untyped().num_allocated_elements() * (dtype == OCU_F64 ? 8 : 4);
  }
};

template <typename T> Grid3DDevice<T> *typed(RefGrid *g);
template <> Grid3DDevice<float> *typed<float>(RefGrid *g) { return g->f; }
template <> Grid3DDevice<double> *typed<double>(RefGrid *g) { return g->d; }

RefGrid *borrow(Grid3DDevice<float> &g) { return new RefGrid{OCU_F32, &g, nullptr, true}; }
RefGrid *borrow(Grid3DDevice<double> &g) { return new RefGrid{OCU_F64, nullptr, &g, true}; }

/* Multigrid solvers behind one handle. */
struct RefMG {
  int kind; /* 0 float, 1 double, 2 reference mixed (double interface) */
  Sol_MultigridPressure3DDevice<float> *f;
  Sol_MultigridPressure3DDevice<double> *d;
  Sol_MultigridPressureMixed3DDeviceD *m;
  RefGrid *pressure;
  Sol_MultigridPressure3DBase *base() {
    return kind == 0 ? (Sol_MultigridPressure3DBase *)f
                     : kind == 1 ? (Sol_MultigridPressure3DBase *)d
                                 : (Sol_MultigridPressure3DBase *)m;
  }
};

void apply_params(Sol_MultigridPressure3DBase *s, const orc_mg_params *p) {
  s->bc = to_bcset(p->bc);
  s->nu1 = p->nu1;
  s->nu2 = p->nu2;
  s->convergence = (ConvergenceType)p->convergence;
  s->make_symmetric_operator = p->make_symmetric_operator != 0;
}

/* Projection solvers behind one handle. */
struct RefProject {
  int kind; /* 0 float, 1 double, 2 double with the reference mixed pressure solver */
  Sol_ProjectDivergence3DDevice<float> *f;
  Sol_ProjectDivergence3DDevice<double> *d;
  Sol_ProjectDivergenceMixed3DDeviceD *m;
  RefGrid *divergence;
  RefGrid *pressure;
};

/* Navier-Stokes equation of either precision. */
struct RefNS {
  int dtype;
  Eqn_IncompressibleNS3D<float> *f;
  Eqn_IncompressibleNS3D<double> *d;
};

template <typename T>
bool ns_set(Eqn_IncompressibleNS3D<T> *eq, const orc_ns_params *p, const void *u, const void *v,
            const void *w, const void *t) {
  Eqn_IncompressibleNS3DParams<T> prm;
  prm.init_grids(p->nx, p->ny, p->nz);
  prm.hx = p->hx;
  prm.hy = p->hy;
  prm.hz = p->hz;
  prm.max_divergence = p->max_divergence;
  prm.temp_bc = to_bcset(p->temp_bc);
  prm.flow_bc = to_bcset(p->flow_bc);
  prm.vertical_direction = (DirectionType)p->vertical_direction;
  prm.gravity = (T)p->gravity;
  prm.bouyancy = (T)p->bouyancy;
  prm.thermal_diffusion = (T)p->thermal_diffusion;
  prm.viscosity = (T)p->viscosity;
  prm.advection_scheme = (InterpolationType)p->advection_scheme;
  prm.time_step = (TimeStepType)p->time_step;
  prm.cfl_factor = p->cfl_factor;
  memcpy(prm.init_u.buffer(), u, sizeof(T) * prm.init_u.num_allocated_elements());
  memcpy(prm.init_v.buffer(), v, sizeof(T) * prm.init_v.num_allocated_elements());
  memcpy(prm.init_w.buffer(), w, sizeof(T) * prm.init_w.num_allocated_elements());
  memcpy(prm.init_temp.buffer(), t, sizeof(T) * prm.init_temp.num_allocated_elements());
  return eq->set_parameters(prm);
}

template <typename T>
const Grid3DDevice<T> *ns_grid(Eqn_IncompressibleNS3D<T> *eq, char which) {
  switch (which) {
    case 'u': return &eq->get_u();
    case 'v': return &eq->get_v();
    case 'w': return &eq->get_w();
    case 't': return &eq->get_temperature();
    default: return nullptr;
  }
}

}  // namespace

extern "C" {

/* ---- grids ------------------------------------------------------------------------------ */

/* A device grid made by Grid3DDevice<T>::init (ocustorage/grid3ddev.cu:358-400). */
void *ref_grid_create(int dtype, int nx, int ny, int nz, int gx, int gy, int gz, int padx,
                      int pady, int padz) {
  if (!ready()) return nullptr;
  RefGrid *g = new RefGrid{dtype, nullptr, nullptr, false};
  bool ok;
  if (dtype == OCU_F64) {
    g->d = new Grid3DDevice<double>();
    ok = g->d->init(nx, ny, nz, gx, gy, gz, padx, pady, padz);
  } else {
    g->f = new Grid3DDevice<float>();
    ok = g->f->init(nx, ny, nz, gx, gy, gz, padx, pady, padz);
  }
  if (!ok) {
    delete g->f;
    delete g->d;
    delete g;
    return nullptr;
  }
  return g;
}

void ref_grid_destroy(void *h) {
  RefGrid *g = (RefGrid *)h;
  if (!g) return;
  if (!g->borrowed) {
    delete g->f;
    delete g->d;
  }
  delete g;
}

void ref_grid_layout(void *h, ocu_layout *out) { fill_layout(((RefGrid *)h)->untyped(), out); }

/* Whole padded buffer, ghosts included, host -> device and back. */
int ref_grid_upload(void *h, const void *host) {
  RefGrid *g = (RefGrid *)h;
  return cudaMemcpy(g->buffer(), host, g->bytes(), cudaMemcpyHostToDevice) == cudaSuccess;
}

int ref_grid_download(void *h, void *host) {
  RefGrid *g = (RefGrid *)h;
  return cudaMemcpy(host, g->buffer(), g->bytes(), cudaMemcpyDeviceToHost) == cudaSuccess;
}

/* ---- multigrid ---------------------------------------------------------------------------- */

/* kind 0/1: Sol_MultigridPressure3DDevice<float/double>; kind 2: the mixed FP64 solver.
 * rhs is borrowed by the solver (sol_mgpressure3ddev.cu:418). */
void *ref_mg_create(int kind, const orc_mg_params *prm, int nx, int ny, int nz, double hx,
                    double hy, double hz, void *rhs) {
  if (!ready()) return nullptr;
  RefGrid *r = (RefGrid *)rhs;
  RefMG *s = new RefMG{kind, nullptr, nullptr, nullptr, nullptr};
  bool ok = false;
  if (kind == 0 && r->dtype == OCU_F32) {
    s->f = new Sol_MultigridPressure3DDevice<float>();
    apply_params(s->f, prm);
    s->f->disable_relax_on_host = prm->disable_relax_on_host != 0;
    ok = s->f->initialize_storage(nx, ny, nz, hx, hy, hz, r->f);
    if (ok) s->pressure = borrow(s->f->pressure());
  } else if (kind == 1 && r->dtype == OCU_F64) {
    s->d = new Sol_MultigridPressure3DDevice<double>();
    apply_params(s->d, prm);
    s->d->disable_relax_on_host = prm->disable_relax_on_host != 0;
    ok = s->d->initialize_storage(nx, ny, nz, hx, hy, hz, r->d);
    if (ok) s->pressure = borrow(s->d->pressure());
  } else if (kind == 2 && r->dtype == OCU_F64) {
    s->m = new Sol_MultigridPressureMixed3DDeviceD();
    apply_params(s->m, prm);
    ok = s->m->initialize_storage(nx, ny, nz, hx, hy, hz, r->d);
    if (ok) s->pressure = borrow(s->m->pressure());
  }
  if (!ok) {
    delete s->f;
    delete s->d;
    delete s->m;
    delete s;
    return nullptr;
  }
  return s;
}

void ref_mg_destroy(void *h) {
  RefMG *s = (RefMG *)h;
  if (!s) return;
  ref_grid_destroy(s->pressure);
  delete s->f;
  delete s->d;
  delete s->m;
  delete s;
}

/* Sol_MultigridPressure3DBase::solve (sol_mgpressure3d.cpp:332-370). */
int ref_mg_solve(void *h, double *residual, double tol, int max_iter) {
  double r = 0;
  bool ok = ((RefMG *)h)->base()->solve(r, tol, max_iter);
  if (residual) *residual = r;
  return ok ? 1 : 0;
}

int ref_mg_run_vcycles(void *h, int count) { return ((RefMG *)h)->base()->run_vcycles(count); }
int ref_mg_run_fmg(void *h, int count) { return ((RefMG *)h)->base()->run_fmg(count); }
void *ref_mg_pressure(void *h) { return ((RefMG *)h)->pressure; }

/* ---- projection --------------------------------------------------------------------------- */

/* kind 0/1: Sol_ProjectDivergence3DDevice<float/double>; kind 2:
 * Sol_ProjectDivergenceMixed3DDeviceD.  u, v, w are borrowed MAC grids of one layout. */
void *ref_project_create(int kind, const ocu_bc_set *bc, int nx, int ny, int nz, double hx,
                         double hy, double hz, void *u, void *v, void *w) {
  if (!ready()) return nullptr;
  RefGrid *U = (RefGrid *)u, *V = (RefGrid *)v, *W = (RefGrid *)w;
  RefProject *p = new RefProject{kind, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool ok = false;
  if (kind == 0) {
    p->f = new Sol_ProjectDivergence3DDevice<float>();
    p->f->bc = to_bcset(*bc);
    ok = p->f->initialize_storage(nx, ny, nz, hx, hy, hz, U->f, V->f, W->f);
    if (ok) {
      p->divergence = borrow(p->f->divergence);
      p->pressure = borrow(p->f->pressure_solver.pressure());
    }
  } else if (kind == 1) {
    p->d = new Sol_ProjectDivergence3DDevice<double>();
    p->d->bc = to_bcset(*bc);
    ok = p->d->initialize_storage(nx, ny, nz, hx, hy, hz, U->d, V->d, W->d);
    if (ok) {
      p->divergence = borrow(p->d->divergence);
      p->pressure = borrow(p->d->pressure_solver.pressure());
    }
  } else if (kind == 2) {
    p->m = new Sol_ProjectDivergenceMixed3DDeviceD();
    p->m->bc = to_bcset(*bc);
    ok = p->m->initialize_storage(nx, ny, nz, hx, hy, hz, U->d, V->d, W->d);
    if (ok) {
      p->divergence = borrow(p->m->divergence);
      p->pressure = borrow(p->m->pressure_solver.pressure());
    }
  }
  if (!ok) {
    delete p->f;
    delete p->d;
    delete p->m;
    delete p;
    return nullptr;
  }
  return p;
}

void ref_project_destroy(void *h) {
  RefProject *p = (RefProject *)h;
  if (!p) return;
  ref_grid_destroy(p->divergence);
  ref_grid_destroy(p->pressure);
  delete p->f;
  delete p->d;
  delete p->m;
  delete p;
}

/* solve(tol): BCs, divergence, pressure to tol in LINF with 15 cycles, gradient, BCs
 * (sol_project3ddev.cu:67-78, sol_projectmixed3d.cu:52-63). */
int ref_project_solve(void *h, double tol) {
  RefProject *p = (RefProject *)h;
  if (p->kind == 0) return p->f->solve(tol);
  if (p->kind == 1) return p->d->solve(tol);
  return p->m->solve(tol);
}

int ref_project_solve_divergence_only(void *h) {
  RefProject *p = (RefProject *)h;
  if (p->kind == 0) return p->f->solve_divergence_only();
  if (p->kind == 1) return p->d->solve_divergence_only();
  return p->m->solve_divergence_only();
}

void *ref_project_divergence(void *h) { return ((RefProject *)h)->divergence; }
void *ref_project_pressure(void *h) { return ((RefProject *)h)->pressure; }

/* ---- advection ---------------------------------------------------------------------------- */

/* One Sol_SelfAdvection3DDevice<T>::solve over borrowed grids (sol_selfadvection3ddev.cu). */
int ref_advect_self(int dtype, int nx, int ny, int nz, double hx, double hy, double hz,
                    int interp, void *u, void *v, void *w, void *dudt, void *dvdt, void *dwdt) {
  if (!ready()) return 0;
  RefGrid *g[6] = {(RefGrid *)u, (RefGrid *)v, (RefGrid *)w,
                   (RefGrid *)dudt, (RefGrid *)dvdt, (RefGrid *)dwdt};
  bool ok;
  if (dtype == OCU_F64) {
    Sol_SelfAdvection3DDevice<double> s;
    s.interp_type = (InterpolationType)interp;
    ok = s.initialize_storage(nx, ny, nz, hx, hy, hz, g[0]->d, g[1]->d, g[2]->d, g[3]->d,
                              g[4]->d, g[5]->d) && s.solve();
  } else {
    Sol_SelfAdvection3DDevice<float> s;
    s.interp_type = (InterpolationType)interp;
    ok = s.initialize_storage(nx, ny, nz, hx, hy, hz, g[0]->f, g[1]->f, g[2]->f, g[3]->f,
                              g[4]->f, g[5]->f) && s.solve();
  }
  return ok && cudaDeviceSynchronize() == cudaSuccess;
}

/* One Sol_PassiveAdvection3DDevice<T>::solve over borrowed grids
 * (sol_passiveadvection3ddev.cu). */
int ref_advect_passive(int dtype, int nx, int ny, int nz, double hx, double hy, double hz,
                       int interp, void *u, void *v, void *w, void *phi, void *dphidt) {
  if (!ready()) return 0;
  RefGrid *g[5] = {(RefGrid *)u, (RefGrid *)v, (RefGrid *)w, (RefGrid *)phi,
                   (RefGrid *)dphidt};
  bool ok;
  if (dtype == OCU_F64) {
    Sol_PassiveAdvection3DDevice<double> s;
    s.interp_type = (InterpolationType)interp;
    ok = s.initialize_storage(nx, ny, nz, hx, hy, hz, g[0]->d, g[1]->d, g[2]->d, g[3]->d,
                              g[4]->d) && s.solve();
  } else {
    Sol_PassiveAdvection3DDevice<float> s;
    s.interp_type = (InterpolationType)interp;
    ok = s.initialize_storage(nx, ny, nz, hx, hy, hz, g[0]->f, g[1]->f, g[2]->f, g[3]->f,
                              g[4]->f) && s.solve();
  }
  return ok && cudaDeviceSynchronize() == cudaSuccess;
}

/* ---- Navier-Stokes ------------------------------------------------------------------------ */

/* Eqn_IncompressibleNS3D<T>::set_parameters (eqn_incompressns3d.cu:164-260) with the initial
 * fields given as host buffers in the layout of Eqn_IncompressibleNS3DParams::init_grids. */
void *ref_ns_create(int dtype, const orc_ns_params *prm, const void *u, const void *v,
                    const void *w, const void *t) {
  if (!ready()) return nullptr;
  RefNS *n = new RefNS{dtype, nullptr, nullptr};
  bool ok;
  if (dtype == OCU_F64) {
    n->d = new Eqn_IncompressibleNS3D<double>();
    ok = ns_set(n->d, prm, u, v, w, t);
  } else {
    n->f = new Eqn_IncompressibleNS3D<float>();
    ok = ns_set(n->f, prm, u, v, w, t);
  }
  if (!ok) {
    delete n->f;
    delete n->d;
    delete n;
    return nullptr;
  }
  return n;
}

void ref_ns_destroy(void *h) {
  RefNS *n = (RefNS *)h;
  if (!n) return;
  delete n->f;
  delete n->d;
  delete n;
}

double ref_ns_get_max_stable_timestep(void *h) {
  RefNS *n = (RefNS *)h;
  return n->dtype == OCU_F64 ? n->d->get_max_stable_timestep() : n->f->get_max_stable_timestep();
}

int ref_ns_advance_one_step(void *h, double dt) {
  RefNS *n = (RefNS *)h;
  return n->dtype == OCU_F64 ? n->d->advance_one_step(dt) : n->f->advance_one_step(dt);
}

/* which: 'u', 'v', 'w', 't'.  Copies the whole padded buffer to host. */
int ref_ns_download(void *h, char which, void *host, ocu_layout *layout_out) {
  RefNS *n = (RefNS *)h;
  if (n->dtype == OCU_F64) {
    const Grid3DDevice<double> *g = ns_grid(n->d, which);
    if (!g) return 0;
    if (layout_out) fill_layout(*g, layout_out);
    return cudaMemcpy(host, g->buffer(), 8 * (size_t)g->num_allocated_elements(),
                      cudaMemcpyDeviceToHost) == cudaSuccess;
  }
  const Grid3DDevice<float> *g = ns_grid(n->f, which);
  if (!g) return 0;
  if (layout_out) fill_layout(*g, layout_out);
  return cudaMemcpy(host, g->buffer(), 4 * (size_t)g->num_allocated_elements(),
                    cudaMemcpyDeviceToHost) == cudaSuccess;
}

/* Sol_PCGPressure3DDevice<T> (sol_pcgpressure3d.cu): rhs and coefficient are reference grids of
 * one layout; the pressure is borrowed from the solver. */
struct RefPCG {
  int dtype;
  Sol_PCGPressure3DDevice<float> *f;
  Sol_PCGPressure3DDevice<double> *d;
  RefGrid *pressure;
};

void *ref_pcg_create(const orc_pcg_params *prm, int nx, int ny, int nz, double hx, double hy, double hz,
                     void *rhs, void *coefficient) {
  if (!ready()) return nullptr;
  RefGrid *r = (RefGrid *)rhs, *c = (RefGrid *)coefficient;
  if (r->dtype != c->dtype) return nullptr;
  RefPCG *s = new RefPCG{r->dtype, nullptr, nullptr, nullptr};
  bool ok;
  if (r->dtype == OCU_F32) {
    s->f = new Sol_PCGPressure3DDevice<float>();
    s->f->bc = to_bcset(prm->bc);
    s->f->convergence = (ConvergenceType)prm->convergence;
    s->f->preconditioner = (PreconditionerType)prm->preconditioner;
    s->f->multigrid_cycles = prm->multigrid_cycles;
    s->f->multigrid_use_fmg = prm->multigrid_use_fmg != 0;
    ok = s->f->initialize_storage(nx, ny, nz, (float)hx, (float)hy, (float)hz, r->f, c->f);
    if (ok) s->pressure = borrow(s->f->pressure());
  } else {
    s->d = new Sol_PCGPressure3DDevice<double>();
    s->d->bc = to_bcset(prm->bc);
    s->d->convergence = (ConvergenceType)prm->convergence;
    s->d->preconditioner = (PreconditionerType)prm->preconditioner;
    s->d->multigrid_cycles = prm->multigrid_cycles;
    s->d->multigrid_use_fmg = prm->multigrid_use_fmg != 0;
    ok = s->d->initialize_storage(nx, ny, nz, (float)hx, (float)hy, (float)hz, r->d, c->d);
    if (ok) s->pressure = borrow(s->d->pressure());
  }
  if (!ok) {
    delete s->f;
    delete s->d;
    delete s;
    return nullptr;
  }
  return s;
}

int ref_pcg_solve(void *h, double *residual, double tol, int max_iter) {
  RefPCG *s = (RefPCG *)h;
  double r = 0;
  const bool ok = s->f ? s->f->solve(r, tol, max_iter) : s->d->solve(r, tol, max_iter);
  cudaDeviceSynchronize();
  *residual = r;
  return ok ? 1 : 0;
}

void *ref_pcg_pressure(void *h) { return ((RefPCG *)h)->pressure; }

void ref_pcg_destroy(void *h) {
  RefPCG *s = (RefPCG *)h;
  if (!s) return;
  ref_grid_destroy(s->pressure);
  delete s->f;
  delete s->d;
  delete s;
}

}  // extern "C"
