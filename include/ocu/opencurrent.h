/*
 * C++ drop-in facade: the OpenCurrent class API (namespace ocu) re-implemented as a header-only
 * layer over the C ABI of libocu_b200.so (ocu_b200.h).  Code written against the reference's
 * headers for the projection-step path compiles against this one:
 *
 *   BoundaryCondition / BoundaryConditionSet     ocuutil/boundary_condition.h:26-112
 *   Grid3DDevice<T> / Grid3DHost<T>               ocustorage/grid3d.h:151-264
 *   apply_3d_(mac_)boundary_conditions_level1*    ocustorage/grid3dboundary.h:26-70
 *   Sol_MultigridPressure3DDevice<T>              ocuequation/sol_mgpressure3d.h:104-181
 *   Sol_MultigridPressure3DDeviceCo<T>            ocuequation/sol_mgpressure3d.h:184-242
 *   Sol_MultigridPressureMixed3DDeviceD           ocuequation/sol_mgpressuremixed3d.h:28-55
 *   Sol_ProjectDivergence3DDevice<T>              ocuequation/sol_project3d.h:74-93
 *   Sol_SelfAdvection3DDevice<T>                  ocuequation/sol_selfadvection3d.h:33-73
 *   Sol_PassiveAdvection3DDevice<T>               ocuequation/sol_passiveadvection3d.h:32-62
 *   Sol_LaplacianCentered3DDevice<T>              ocuequation/sol_laplaciancent3d.h:28-58
 *   Eqn_IncompressibleNS3DParams<T> / Eqn_IncompressibleNS3D<T>
 *                                                 ocuequation/eqn_incompressns3d.h:34-177
 *
 * Conventions kept from the reference: bool returns, solve(double &residual, tol, max_iter),
 * public fields (bc, nu1, nu2, convergence, make_symmetric_operator, disable_relax_on_host),
 * borrowed rhs / velocity grids, non-copyable grids.  Errors print the library's message and
 * set the sticky any_error() flag (ocuequation/error_handler.h:27-57).  All work is enqueued on
 * the stream passed to set_stream() (default: the legacy default stream).
 */
#ifndef OCU_OPENCURRENT_H
#define OCU_OPENCURRENT_H

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../ocu_b200.h"

namespace ocu {

enum BoundaryConditionType {
  BC_INVALID = OCU_BC_INVALID, BC_NONE = OCU_BC_NONE, BC_PERIODIC = OCU_BC_PERIODIC,
  BC_DIRICHELET = OCU_BC_DIRICHELET, BC_NEUMANN = OCU_BC_NEUMANN, BC_SECOND_DERIV = OCU_BC_SECOND_DERIV,
  BC_DIRICHELET_AND_NEUMANN = OCU_BC_DIRICHELET_AND_NEUMANN,
  BC_FORCED_INFLOW_VARIABLE_SLIP = OCU_BC_FORCED_INFLOW_VARIABLE_SLIP, BC_SCALAR_SLIP = OCU_BC_SCALAR_SLIP
};

enum ConvergenceType {
  CONVERGENCE_CALC_L2 = OCU_CONVERGENCE_CALC_L2, CONVERGENCE_CALC_LINF = OCU_CONVERGENCE_CALC_LINF,
  CONVERGENCE_CRITERIA_L2 = OCU_CONVERGENCE_CRITERIA_L2, CONVERGENCE_CRITERIA_LINF = OCU_CONVERGENCE_CRITERIA_LINF,
  CONVERGENCE_CRITERIA_NONE = OCU_CONVERGENCE_CRITERIA_NONE, CONVERGENCE_L2 = OCU_CONVERGENCE_L2,
  CONVERGENCE_LINF = OCU_CONVERGENCE_LINF, CONVERGENCE_NONE = OCU_CONVERGENCE_NONE,
  CONVERGENCE_NONE_CALC_L2LINF = OCU_CONVERGENCE_NONE_CALC_L2LINF
};

enum InterpolationType {
  IT_ERROR = OCU_IT_ERROR, IT_FIRST_ORDER_UPWIND = OCU_IT_FIRST_ORDER_UPWIND,
  IT_SECOND_ORDER_CENTERED = OCU_IT_SECOND_ORDER_CENTERED,
  IT_THIRD_ORDER_VAN_LEER_FLUX_LIMITED = OCU_IT_THIRD_ORDER_VAN_LEER_FLUX_LIMITED
};

enum PreconditionerType {
  PRECOND_NONE = OCU_PRECOND_NONE, PRECOND_JACOBI = OCU_PRECOND_JACOBI,
  PRECOND_MULTIGRID = OCU_PRECOND_MULTIGRID, PRECOND_BFBT = OCU_PRECOND_BFBT
};
enum GridStaggering {
  GS_CENTER_POINT = OCU_GS_CENTER_POINT, GS_U_FACE = OCU_GS_U_FACE, GS_V_FACE = OCU_GS_V_FACE,
  GS_W_FACE = OCU_GS_W_FACE, GS_CUSTOM = OCU_GS_CUSTOM
};
typedef int nc_type;
enum { NC_INT = OCU_NC_INT, NC_FLOAT = OCU_NC_FLOAT, NC_DOUBLE = OCU_NC_DOUBLE };
enum TimeStepType { TS_ERROR = OCU_TS_ERROR, TS_FORWARD_EULER = OCU_TS_FORWARD_EULER, TS_ADAMS_BASHFORD2 = OCU_TS_ADAMS_BASHFORD2 };

enum DirectionType {
  DIR_POSITIVE_FLAG = OCU_DIR_POSITIVE_FLAG, DIR_NEGATIVE_FLAG = OCU_DIR_NEGATIVE_FLAG,
  DIR_XAXIS_FLAG = OCU_DIR_XAXIS_FLAG, DIR_YAXIS_FLAG = OCU_DIR_YAXIS_FLAG, DIR_ZAXIS_FLAG = OCU_DIR_ZAXIS_FLAG,
  DIR_XPOS = OCU_DIR_XPOS, DIR_XNEG = OCU_DIR_XNEG, DIR_YPOS = OCU_DIR_YPOS, DIR_YNEG = OCU_DIR_YNEG,
  DIR_ZPOS = OCU_DIR_ZPOS, DIR_ZNEG = OCU_DIR_ZNEG
};

struct BoundaryCondition {
  BoundaryConditionType type;
  float value;
  float aux_value;
  BoundaryCondition() : type(BC_INVALID), value(0), aux_value(0) {}
  bool check_type(BoundaryConditionType t) const { return t == type; }
  ocu_bc c() const { ocu_bc b; b.type = type; b.value = value; b.aux_value = aux_value; return b; }
};

struct BoundaryConditionSet {
  BoundaryCondition xpos, xneg, ypos, yneg, zpos, zneg;
  BoundaryConditionSet() {}
  explicit BoundaryConditionSet(const BoundaryCondition &v) : xpos(v), xneg(v), ypos(v), yneg(v), zpos(v), zneg(v) {}
  void make_homogeneous() {
    BoundaryCondition *f[6] = {&xpos, &xneg, &ypos, &yneg, &zpos, &zneg};
    for (int i = 0; i < 6; i++) f[i]->value = f[i]->aux_value = 0;
  }
  ocu_bc_set c() const {
    ocu_bc_set s;
    s.xpos = xpos.c(); s.xneg = xneg.c(); s.ypos = ypos.c(); s.yneg = yneg.c(); s.zpos = zpos.c(); s.zneg = zneg.c();
    return s;
  }
};

// Sticky error flag of the reference's ErrorHandler.
class ErrorHandler {
  bool _any_error = false;
 protected:
  bool check_ok(ocu_status st, const char *what = nullptr) {
    if (st != OCU_OK) {
      std::printf("%s%s%s\n", what ? what : "", what ? ": " : "", ocu_last_error());
      _any_error = true;
      return false;
    }
    return true;
  }
 public:
  void add_error() { _any_error = true; }
  void clear_error() { _any_error = false; }
  bool any_error() const { return _any_error; }
};

namespace detail {
template <typename T> struct dtype_of;
template <> struct dtype_of<float> { static const ocu_dtype value = OCU_F32; };
template <> struct dtype_of<double> { static const ocu_dtype value = OCU_F64; };
inline ocu_stream &stream() { static ocu_stream s = nullptr; return s; }
}  // namespace detail

// Stream used by every facade call (ThreadManager::get_compute_stream in the reference).
inline void set_stream(ocu_stream s) { detail::stream() = s; }

template <typename T> class Grid3DDevice;

// Host grid in the same padded layout (pinned flag accepted, allocation is pageable here).
template <typename T>
class Grid3DHost {
  ocu_layout _L;
  std::vector<T> _buf;
  Grid3DHost(const Grid3DHost &);
  Grid3DHost &operator=(const Grid3DHost &);
 public:
  Grid3DHost() { std::memset(&_L, 0, sizeof(_L)); }
  bool init(int nx, int ny, int nz, int gx, int gy, int gz, bool pinned = true, int padx = 0, int pady = 0, int padz = 0) {
    (void)pinned;
    if (ocu_layout_compute(nx, ny, nz, gx, gy, gz, padx, pady, padz, &_L) != OCU_OK) return false;
    _buf.assign((size_t)_L.allocated, (T)0);
    return true;
  }
  template <typename G> bool init_congruent(const G &o, bool pinned = true) {
    return init(o.nx(), o.ny(), o.nz(), o.gx(), o.gy(), o.gz(), pinned, o.paddingx(), o.paddingy(), o.paddingz());
  }
  int nx() const { return _L.nx; } int ny() const { return _L.ny; } int nz() const { return _L.nz; }
  int gx() const { return _L.gx; } int gy() const { return _L.gy; } int gz() const { return _L.gz; }
  int pnx() const { return _L.pnx; } int pny() const { return _L.pny; } int pnz() const { return _L.pnz; }
  int paddingx() const { return _L.pnx - (_L.nx + 2 * _L.gx); }
  int paddingy() const { return _L.pny - (_L.ny + 2 * _L.gy); }
  int paddingz() const { return _L.pnz - (_L.nz + 2 * _L.gz); }
  int xstride() const { return _L.xstride; } int ystride() const { return _L.ystride; }
  int num_allocated_elements() const { return (int)_L.allocated; }
  T &at(int i, int j, int k) { return _buf[(size_t)(_L.shift + (long long)i * _L.xstride + (long long)j * _L.ystride + k)]; }
  const T &at(int i, int j, int k) const { return _buf[(size_t)(_L.shift + (long long)i * _L.xstride + (long long)j * _L.ystride + k)]; }
  T *buffer() { return _buf.data(); }
  const T *buffer() const { return _buf.data(); }
  void clear_zero() { std::fill(_buf.begin(), _buf.end(), (T)0); }
  bool copy_all_data(const Grid3DDevice<T> &from);
};

template <typename T>
class Grid3DDevice {
  ocu_grid *_g = nullptr;
  bool _own = true;
  Grid3DDevice(const Grid3DDevice &);
  Grid3DDevice &operator=(const Grid3DDevice &);
  ocu_layout L() const { ocu_layout l; std::memset(&l, 0, sizeof(l)); if (_g) ocu_grid_info(_g, &l, nullptr, nullptr); return l; }
 public:
  Grid3DDevice() {}
  ~Grid3DDevice() { if (_own) ocu_grid_destroy(_g); }
  // wrap a handle owned by a solver (read_u/read_r/read_b/pressure)
  void attach(ocu_grid *g) { if (_own) ocu_grid_destroy(_g); _g = g; _own = false; }
  ocu_grid *handle() const { return _g; }
  bool init(int nx, int ny, int nz, int gx, int gy, int gz, int padx = 0, int pady = 0, int padz = 0) {
    if (_own) ocu_grid_destroy(_g);
    _own = true;
    return ocu_grid_create(detail::dtype_of<T>::value, nx, ny, nz, gx, gy, gz, padx, pady, padz, &_g) == OCU_OK;
  }
  template <typename G> bool init_congruent(const G &o) {
    return init(o.nx(), o.ny(), o.nz(), o.gx(), o.gy(), o.gz(), o.paddingx(), o.paddingy(), o.paddingz());
  }
  int nx() const { return L().nx; } int ny() const { return L().ny; } int nz() const { return L().nz; }
  int gx() const { return L().gx; } int gy() const { return L().gy; } int gz() const { return L().gz; }
  int pnx() const { return L().pnx; } int pny() const { return L().pny; } int pnz() const { return L().pnz; }
  int paddingx() const { ocu_layout l = L(); return l.pnx - (l.nx + 2 * l.gx); }
  int paddingy() const { ocu_layout l = L(); return l.pny - (l.ny + 2 * l.gy); }
  int paddingz() const { ocu_layout l = L(); return l.pnz - (l.nz + 2 * l.gz); }
  int xstride() const { return L().xstride; } int ystride() const { return L().ystride; }
  int shift_amount() const { return (int)L().shift; }
  int num_allocated_elements() const { return (int)L().allocated; }
  T *buffer() { void *p = nullptr; ocu_grid_info(_g, nullptr, nullptr, &p); return (T *)p; }
  const T *buffer() const { void *p = nullptr; ocu_grid_info(_g, nullptr, nullptr, &p); return (const T *)p; }
  bool check_layout_match(const Grid3DDevice &o) const { return pnx() == o.pnx() && pny() == o.pny() && pnz() == o.pnz(); }
  bool check_interior_dimension_match(const Grid3DDevice &o) const { return nx() == o.nx() && ny() == o.ny() && nz() == o.nz(); }
  bool clear_zero() { return ocu_grid_clear(_g, 0.0, detail::stream()) == OCU_OK; }
  bool clear(T t) { return ocu_grid_clear(_g, (double)t, detail::stream()) == OCU_OK; }
  template <typename S> bool copy_all_data(const Grid3DDevice<S> &from) {
    return ocu_grid_copy_all_data(_g, from.handle(), detail::stream()) == OCU_OK;
  }
  bool copy_all_data(const Grid3DHost<T> &from) { return ocu_grid_upload(_g, from.buffer(), detail::stream()) == OCU_OK; }
  bool linear_combination(T a1, const Grid3DDevice &g1) {
    return ocu_grid_linear_combination(_g, (double)a1, g1._g, 0.0, nullptr, detail::stream()) == OCU_OK;
  }
  bool linear_combination(T a1, const Grid3DDevice &g1, T a2, const Grid3DDevice &g2) {
    return ocu_grid_linear_combination(_g, (double)a1, g1._g, (double)a2, g2._g, detail::stream()) == OCU_OK;
  }
  bool reduce(ocu_reduce_op op, T &result) const {
    double r = 0;
    if (ocu_grid_reduce(_g, op, &r, detail::stream()) != OCU_OK) return false;
    result = (T)r;
    return true;
  }
  bool reduce_maxabs(T &r) const { return reduce(OCU_REDUCE_MAXABS, r); }
  bool reduce_max(T &r) const { return reduce(OCU_REDUCE_MAX, r); }
  bool reduce_min(T &r) const { return reduce(OCU_REDUCE_MIN, r); }
  bool reduce_sum(T &r) const { return reduce(OCU_REDUCE_SUM, r); }
  bool reduce_sqrsum(T &r) const { return reduce(OCU_REDUCE_SQRSUM, r); }
  bool reduce_checknan(T &r) const { return reduce(OCU_REDUCE_CHECKNAN, r); }
};

template <typename T>
bool Grid3DHost<T>::copy_all_data(const Grid3DDevice<T> &from) {
  return ocu_grid_download(from.handle(), _buf.data(), detail::stream()) == OCU_OK;
}

typedef Grid3DDevice<float> Grid3DDeviceF;
typedef Grid3DDevice<double> Grid3DDeviceD;
typedef Grid3DHost<float> Grid3DHostF;
typedef Grid3DHost<double> Grid3DHostD;

template <typename T>
bool apply_3d_boundary_conditions_level1(Grid3DDevice<T> &g, const BoundaryConditionSet &bc, double hx, double hy, double hz) {
  ocu_bc_set s = bc.c();
  return ocu_apply_boundary_conditions(g.handle(), &s, hx, hy, hz, OCU_BC_LEVEL1, detail::stream()) == OCU_OK;
}
template <typename T>
bool apply_3d_boundary_conditions_level1_nocorners(Grid3DDevice<T> &g, const BoundaryConditionSet &bc, double hx, double hy, double hz) {
  ocu_bc_set s = bc.c();
  return ocu_apply_boundary_conditions(g.handle(), &s, hx, hy, hz, OCU_BC_LEVEL1_NOCORNERS, detail::stream()) == OCU_OK;
}
template <typename T>
bool apply_3d_mac_boundary_conditions_level1(Grid3DDevice<T> &u, Grid3DDevice<T> &v, Grid3DDevice<T> &w,
                                             const BoundaryConditionSet &bc, double hx, double hy, double hz) {
  ocu_bc_set s = bc.c();
  return ocu_apply_mac_boundary_conditions(u.handle(), v.handle(), w.handle(), &s, hx, hy, hz, detail::stream()) == OCU_OK;
}

// ---- multigrid --------------------------------------------------------------------------
class Sol_MultigridPressure3DBase : public ErrorHandler {
 protected:
  ocu_mg *_mg = nullptr;
  ocu_mg_kind _kind;
  ocu_mg_params params() const {
    ocu_mg_params p;
    ocu_mg_params_default(&p);
    p.bc = bc.c();
    p.nu1 = nu1; p.nu2 = nu2;
    p.convergence = convergence;
    p.make_symmetric_operator = make_symmetric_operator ? 1 : 0;
    p.disable_relax_on_host = disable_relax_on_host ? 1 : 0;
    return p;
  }
  bool sync_params() {
    ocu_mg_params p = params();
    return check_ok(ocu_mg_set_params(_mg, &p));
  }
 public:
  BoundaryConditionSet bc;
  int nu1 = 2, nu2 = 2;
  ConvergenceType convergence = CONVERGENCE_L2;
  bool make_symmetric_operator = false;
  bool disable_relax_on_host = false;

  explicit Sol_MultigridPressure3DBase(ocu_mg_kind k) : _kind(k) {}
  ~Sol_MultigridPressure3DBase() { ocu_mg_destroy(_mg); }
  ocu_mg *handle() const { return _mg; }

  bool solve(double &residual, double tolerance = 1e-6, int max_iter = 4) {
    if (!sync_params()) return false;
    ocu_stream s = detail::stream();
    ocu_mg_set_stream(_mg, s);
    ocu_status st = ocu_mg_solve(_mg, &residual, tolerance, max_iter);
    if (st == OCU_ERR_NOT_CONVERGED) return false;
    return check_ok(st, "[WARNING] Sol_MultigridPressure3DBase::solve");
  }
  bool run_vcycles(int count) { return sync_params() && check_ok(ocu_mg_run_vcycles(_mg, count)); }
  bool run_fmg(int count) { return sync_params() && check_ok(ocu_mg_run_fmg(_mg, count)); }
};

template <typename T>
class Sol_MultigridPressure3DDevice : public Sol_MultigridPressure3DBase {
  Grid3DDevice<T> _pressure;
  mutable Grid3DDevice<T> _view;
 public:
  Sol_MultigridPressure3DDevice() : Sol_MultigridPressure3DBase(sizeof(T) == 8 ? OCU_MG_F64 : OCU_MG_F32) {}
  bool initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, Grid3DDevice<T> *rhs) {
    ocu_mg_params p = params();
    if (!check_ok(ocu_mg_create(_kind, &p, &_mg))) return false;
    ocu_mg_set_stream(_mg, detail::stream());
    if (!check_ok(ocu_mg_initialize_storage(_mg, nx, ny, nz, hx, hy, hz, rhs->handle()))) return false;
    _pressure.attach(ocu_mg_pressure(_mg));
    return true;
  }
  Grid3DDevice<T> &pressure() { return _pressure; }
  const Grid3DDevice<T> &pressure() const { return _pressure; }
  const Grid3DDevice<T> &read_u(int level) const { _view.attach(ocu_mg_level_grid(_mg, 'u', level)); return _view; }
  const Grid3DDevice<T> &read_r(int level) const { _view.attach(ocu_mg_level_grid(_mg, 'r', level)); return _view; }
  const Grid3DDevice<T> &read_b(int level) const { _view.attach(ocu_mg_level_grid(_mg, 'b', level)); return _view; }
};

typedef Sol_MultigridPressure3DDevice<float> Sol_MultigridPressure3DDeviceF;
typedef Sol_MultigridPressure3DDevice<double> Sol_MultigridPressure3DDeviceD;

// Sol_MultigridPressure3DDeviceCo<T> (sol_mgpressure3d.h:184-242).  The reference builds one
// object per image thread; here one object drives all `num_images` slabs (image i on
// devices[i], several images may share a device).  initialize_storage takes the slab size along
// x and one rhs per image; co_pressure(i) is image i's slab of the pressure.  solve / run_vcycles
// / run_fmg and the parameters are Sol_MultigridPressure3DBase's.
template <typename T>
class Sol_MultigridPressure3DDeviceCo : public Sol_MultigridPressure3DBase {
  std::string _id;
  int _images;
  std::vector<int> _devices;
  std::unique_ptr<Grid3DDevice<T>[]> _co_pressure;
 public:
  long long grid_size_for_cutoff = 64 * 64 * 64;  // sol_mgpressure3dco.cu:223
  Sol_MultigridPressure3DDeviceCo(const char *id, int num_images, const int *devices = nullptr)
      : Sol_MultigridPressure3DBase(sizeof(T) == 8 ? OCU_MG_F64 : OCU_MG_F32), _id(id ? id : ""),
        _images(num_images), _devices(num_images > 0 ? num_images : 0, 0) {
    if (devices)
      for (int i = 0; i < num_images; i++) _devices[i] = devices[i];
  }
  bool initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, Grid3DDevice<T> *const *rhs) {
    ocu_mg_params p = params();
    if (!check_ok(ocu_mgco_create(_kind, &p, _images, _devices.data(), &_mg))) return false;
    ocu_mg_set_stream(_mg, detail::stream());
    if (!check_ok(ocu_mgco_set_cutoff_cells(_mg, grid_size_for_cutoff))) return false;
    std::vector<ocu_grid *> h(_images);
    for (int i = 0; i < _images; i++) h[i] = rhs[i]->handle();
    if (!check_ok(ocu_mgco_initialize_storage(_mg, nx, ny, nz, hx, hy, hz, h.data()))) return false;
    _co_pressure.reset(new Grid3DDevice<T>[_images]);
    for (int i = 0; i < _images; i++) _co_pressure[i].attach(ocu_mgco_pressure(_mg, i));
    return true;
  }
  int num_images() const { return _images; }
  int cutoff_level() const { return ocu_mgco_cutoff_level(_mg); }
  Grid3DDevice<T> &co_pressure(int image) { return _co_pressure[image]; }
  const Grid3DDevice<T> &co_pressure(int image) const { return _co_pressure[image]; }
};

// FP64 interface; the default algorithm is FP32 V-cycles inside FP64 iterative refinement,
// use_reference_algorithm() selects the reference FP32 warm start + FP64 FMG.
class Sol_MultigridPressureMixed3DDeviceD : public Sol_MultigridPressure3DBase {
  Grid3DDevice<double> _pressure;
 public:
  Sol_MultigridPressureMixed3DDeviceD() : Sol_MultigridPressure3DBase(OCU_MG_MIXED_IR) {}
  void use_reference_algorithm(bool on = true) { _kind = on ? OCU_MG_MIXED_WARMSTART : OCU_MG_MIXED_IR; }
  bool initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, Grid3DDevice<double> *rhs) {
    ocu_mg_params p = params();
    if (!check_ok(ocu_mg_create(_kind, &p, &_mg))) return false;
    ocu_mg_set_stream(_mg, detail::stream());
    if (!check_ok(ocu_mg_initialize_storage(_mg, nx, ny, nz, hx, hy, hz, rhs->handle()))) return false;
    _pressure.attach(ocu_mg_pressure(_mg));
    return true;
  }
  Grid3DDevice<double> &pressure() { return _pressure; }
};

// ---- projection and stencils ----------------------------------------------------------------
template <typename T>
class Sol_ProjectDivergence3DDevice : public ErrorHandler {
  ocu_project *_p = nullptr;
  Grid3DDevice<T> _div;
 public:
  BoundaryConditionSet bc;
  Grid3DDevice<T> *u = nullptr, *v = nullptr, *w = nullptr;
  Sol_ProjectDivergence3DDevice() { ocu_project_create(detail::dtype_of<T>::value, &_p); }
  ~Sol_ProjectDivergence3DDevice() { ocu_project_destroy(_p); }
  bool initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, Grid3DDevice<T> *u_,
                          Grid3DDevice<T> *v_, Grid3DDevice<T> *w_) {
    u = u_; v = v_; w = w_;
    ocu_bc_set s = bc.c();
    ocu_project_set_stream(_p, detail::stream());
    if (!check_ok(ocu_project_initialize_storage(_p, nx, ny, nz, hx, hy, hz, u->handle(), v->handle(), w->handle(), &s)))
      return false;
    _div.attach(ocu_project_divergence(_p));
    return true;
  }
  bool solve(double tolerance = 1e-5) {
    clear_error();
    ocu_status st = ocu_project_solve(_p, tolerance);
    if (st == OCU_ERR_NOT_CONVERGED) { add_error(); return false; }
    return check_ok(st);
  }
  bool solve_divergence_only() { clear_error(); return check_ok(ocu_project_solve_divergence_only(_p)); }
  Grid3DDevice<T> &divergence() { return _div; }
};

typedef Sol_ProjectDivergence3DDevice<float> Sol_ProjectDivergence3DDeviceF;
typedef Sol_ProjectDivergence3DDevice<double> Sol_ProjectDivergence3DDeviceD;

// Sol_ProjectDivergenceMixed3DDeviceD (sol_projectmixed3d.h:28-45): FP64 fields, mixed-precision
// pressure solver.  As for Sol_MultigridPressureMixed3DDeviceD, the default pressure algorithm is
// FP32 V-cycles inside FP64 iterative refinement; use_reference_algorithm() (before
// initialize_storage) selects the reference's FP32 warm start + FP64 FMG.
class Sol_ProjectDivergenceMixed3DDeviceD : public ErrorHandler {
  ocu_project *_p = nullptr;
  ocu_mg_kind _kind = OCU_MG_MIXED_IR;
  Grid3DDevice<double> _div;
 public:
  BoundaryConditionSet bc;
  Grid3DDevice<double> *u = nullptr, *v = nullptr, *w = nullptr;
  ~Sol_ProjectDivergenceMixed3DDeviceD() { ocu_project_destroy(_p); }
  void use_reference_algorithm(bool on = true) { _kind = on ? OCU_MG_MIXED_WARMSTART : OCU_MG_MIXED_IR; }
  bool initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, Grid3DDevice<double> *u_,
                          Grid3DDevice<double> *v_, Grid3DDevice<double> *w_) {
    u = u_; v = v_; w = w_;
    if (!_p && !check_ok(ocu_project_create_with(_kind, &_p))) return false;
    ocu_bc_set s = bc.c();
    ocu_project_set_stream(_p, detail::stream());
    if (!check_ok(ocu_project_initialize_storage(_p, nx, ny, nz, hx, hy, hz, u->handle(), v->handle(), w->handle(), &s)))
      return false;
    _div.attach(ocu_project_divergence(_p));
    return true;
  }
  bool solve(double tolerance = 1e-5) {
    clear_error();
    ocu_status st = ocu_project_solve(_p, tolerance);
    if (st == OCU_ERR_NOT_CONVERGED) { add_error(); return false; }
    return check_ok(st);
  }
  bool solve_divergence_only() { clear_error(); return check_ok(ocu_project_solve_divergence_only(_p)); }
  Grid3DDevice<double> &divergence() { return _div; }
};

template <typename T>
class Sol_SelfAdvection3DDevice : public ErrorHandler {
  int _nx = 0, _ny = 0, _nz = 0;
  double _hx = 0, _hy = 0, _hz = 0;
 public:
  InterpolationType interp_type = IT_FIRST_ORDER_UPWIND;
  Grid3DDevice<T> *u = nullptr, *v = nullptr, *w = nullptr, *deriv_udt = nullptr, *deriv_vdt = nullptr, *deriv_wdt = nullptr;
  bool initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, Grid3DDevice<T> *u_, Grid3DDevice<T> *v_,
                          Grid3DDevice<T> *w_, Grid3DDevice<T> *du, Grid3DDevice<T> *dv, Grid3DDevice<T> *dw) {
    _nx = nx; _ny = ny; _nz = nz; _hx = hx; _hy = hy; _hz = hz;
    u = u_; v = v_; w = w_; deriv_udt = du; deriv_vdt = dv; deriv_wdt = dw;
    return u->nx() == nx + 1 && v->ny() == ny + 1 && w->nz() == nz + 1 && u->check_layout_match(*v) && u->check_layout_match(*w);
  }
  bool solve() {
    return check_ok(ocu_advect_self(u->handle(), v->handle(), w->handle(), deriv_udt->handle(), deriv_vdt->handle(),
                                    deriv_wdt->handle(), _nx, _ny, _nz, _hx, _hy, _hz, (ocu_interpolation)interp_type,
                                    detail::stream()));
  }
};

template <typename T>
class Sol_PassiveAdvection3DDevice : public ErrorHandler {
  int _nx = 0, _ny = 0, _nz = 0;
  double _hx = 0, _hy = 0, _hz = 0;
 public:
  InterpolationType interp_type = IT_FIRST_ORDER_UPWIND;
  Grid3DDevice<T> *u = nullptr, *v = nullptr, *w = nullptr, *phi = nullptr, *deriv_phidt = nullptr;
  bool initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, Grid3DDevice<T> *u_, Grid3DDevice<T> *v_,
                          Grid3DDevice<T> *w_, Grid3DDevice<T> *phi_, Grid3DDevice<T> *dphi) {
    _nx = nx; _ny = ny; _nz = nz; _hx = hx; _hy = hy; _hz = hz;
    u = u_; v = v_; w = w_; phi = phi_; deriv_phidt = dphi;
    return true;
  }
  bool solve() {
    return check_ok(ocu_advect_passive(u->handle(), v->handle(), w->handle(), phi->handle(), deriv_phidt->handle(), _nx,
                                       _ny, _nz, _hx, _hy, _hz, (ocu_interpolation)interp_type, detail::stream()));
  }
};

template <typename T>
class Sol_LaplacianCentered3DDevice : public ErrorHandler {
  int _nx = 0, _ny = 0, _nz = 0;
  double _hx = 0, _hy = 0, _hz = 0;
 public:
  T coefficient = 1;
  Grid3DDevice<T> *phi = nullptr, *deriv_phidt = nullptr;
  bool initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, Grid3DDevice<T> *phi_, Grid3DDevice<T> *dphi) {
    _nx = nx; _ny = ny; _nz = nz; _hx = hx; _hy = hy; _hz = hz;
    phi = phi_; deriv_phidt = dphi;
    return phi->check_layout_match(*dphi);
  }
  bool solve() {
    return check_ok(ocu_laplacian_add(phi->handle(), deriv_phidt->handle(), _nx, _ny, _nz, _hx, _hy, _hz,
                                      (double)coefficient, detail::stream()));
  }
};

// ---- Navier-Stokes --------------------------------------------------------------------------
template <typename T>
class Eqn_IncompressibleNS3DParams {
 public:
  int nx = 0, ny = 0, nz = 0;
  double hx = 0, hy = 0, hz = 0;
  double max_divergence = 1e-5;
  BoundaryConditionSet temp_bc, flow_bc;
  DirectionType vertical_direction = DIR_YPOS;
  T gravity = (T)-9.8, bouyancy = 1;
  Grid3DHost<T> init_u, init_v, init_w, init_temp;
  T thermal_diffusion = 0, viscosity = 0;
  InterpolationType advection_scheme = IT_FIRST_ORDER_UPWIND;
  TimeStepType time_step = TS_FORWARD_EULER;
  double cfl_factor = 1;
  // not a reference field: the projection's pressure solved by FP32 V-cycles in FP64 refinement
  bool mixed_pressure = false;
  void init_grids(int nx_, int ny_, int nz_, bool pinned = true) {
    nx = nx_; ny = ny_; nz = nz_;
    init_u.init(nx + 1, ny, nz, 1, 1, 1, pinned, 0, 1, 1);
    init_v.init(nx, ny + 1, nz, 1, 1, 1, pinned, 1, 0, 1);
    init_w.init(nx, ny, nz + 1, 1, 1, 1, pinned, 1, 1, 0);
    init_temp.init(nx, ny, nz, 1, 1, 1, pinned, 1, 1, 1);
  }
};

template <typename T>
class Eqn_IncompressibleNS3D : public ErrorHandler {
  ocu_ns *_ns = nullptr;
  mutable Grid3DDevice<T> _g[4];
 public:
  int num_steps() const { return ocu_ns_num_steps(_ns); }
  Eqn_IncompressibleNS3D() { ocu_ns_create(detail::dtype_of<T>::value, &_ns); }
  ~Eqn_IncompressibleNS3D() { ocu_ns_destroy(_ns); }
  bool set_parameters(const Eqn_IncompressibleNS3DParams<T> &p) {
    ocu_ns_params c;
    ocu_ns_params_default(&c);
    c.nx = p.nx; c.ny = p.ny; c.nz = p.nz;
    c.hx = p.hx; c.hy = p.hy; c.hz = p.hz;
    c.max_divergence = p.max_divergence;
    c.temp_bc = p.temp_bc.c();
    c.flow_bc = p.flow_bc.c();
    c.vertical_direction = p.vertical_direction;
    c.gravity = (double)p.gravity; c.bouyancy = (double)p.bouyancy;
    c.thermal_diffusion = (double)p.thermal_diffusion; c.viscosity = (double)p.viscosity;
    c.advection_scheme = p.advection_scheme; c.time_step = p.time_step; c.cfl_factor = p.cfl_factor;
    c.mixed_pressure = p.mixed_pressure ? 1 : 0;
    ocu_ns_set_stream(_ns, detail::stream());
    return check_ok(ocu_ns_set_parameters(_ns, &c, p.init_u.buffer(), p.init_v.buffer(), p.init_w.buffer(), p.init_temp.buffer()));
  }
  double get_max_stable_timestep() const {
    double dt = 0;
    ocu_ns_get_max_stable_timestep(_ns, &dt);
    return dt;
  }
  bool advance_one_step(double dt) {
    clear_error();
    ocu_status st = ocu_ns_advance_one_step(_ns, dt);
    if (st == OCU_ERR_NOT_CONVERGED) { add_error(); return false; }
    return check_ok(st);
  }
  bool advance(double dt) {
    ocu_status st = ocu_ns_advance(_ns, dt);
    if (st == OCU_ERR_NOT_CONVERGED) return false;
    return check_ok(st);
  }
  const Grid3DDevice<T> &get_u() const { _g[0].attach(ocu_ns_grid(_ns, 'u')); return _g[0]; }
  const Grid3DDevice<T> &get_v() const { _g[1].attach(ocu_ns_grid(_ns, 'v')); return _g[1]; }
  const Grid3DDevice<T> &get_w() const { _g[2].attach(ocu_ns_grid(_ns, 'w')); return _g[2]; }
  const Grid3DDevice<T> &get_temperature() const { _g[3].attach(ocu_ns_grid(_ns, 't')); return _g[3]; }
};

typedef Eqn_IncompressibleNS3D<float> Eqn_IncompressibleNS3DF;
typedef Eqn_IncompressibleNS3D<double> Eqn_IncompressibleNS3DD;
typedef Eqn_IncompressibleNS3DParams<float> Eqn_IncompressibleNS3DParamsF;
typedef Eqn_IncompressibleNS3DParams<double> Eqn_IncompressibleNS3DParamsD;

// Sol_PCGPressure3DDevice<T> (sol_pcgpressure3d.h:41-97): conjugate gradients on
// -div(coefficient grad p) = rhs; the public fields are read at initialize_storage and at each
// solve (bc only at initialize_storage).
template <typename T>
class Sol_PCGPressure3DDevice : public ErrorHandler {
  ocu_pcg *_s = nullptr;
  Grid3DDevice<T> _pressure;
  ocu_pcg_params params() const {
    ocu_pcg_params p;
    ocu_pcg_params_default(&p);
    p.bc = bc.c();
    p.convergence = convergence;
    p.preconditioner = preconditioner;
    p.multigrid_cycles = multigrid_cycles;
    p.multigrid_use_fmg = multigrid_use_fmg ? 1 : 0;
    return p;
  }
 public:
  BoundaryConditionSet bc;
  ConvergenceType convergence = CONVERGENCE_L2;
  PreconditionerType preconditioner = PRECOND_BFBT;
  int multigrid_cycles = 2;
  bool multigrid_use_fmg = true;
  Grid3DDevice<T> *rhs_grid = nullptr, *coefficient_grid = nullptr;
  ~Sol_PCGPressure3DDevice() { ocu_pcg_destroy(_s); }
  bool initialize_storage(int nx, int ny, int nz, float hx, float hy, float hz, Grid3DDevice<T> *rhs,
                          Grid3DDevice<T> *coefficient) {
    rhs_grid = rhs;
    coefficient_grid = coefficient;
    ocu_pcg_params p = params();
    if (!_s && !check_ok(ocu_pcg_create(detail::dtype_of<T>::value, &p, &_s))) return false;
    ocu_pcg_set_stream(_s, detail::stream());
    if (!check_ok(ocu_pcg_initialize_storage(_s, nx, ny, nz, hx, hy, hz, rhs->handle(), coefficient->handle())))
      return false;
    ocu_grid *g = nullptr;
    if (!check_ok(ocu_pcg_pressure(_s, &g))) return false;
    _pressure.attach(g);
    return true;
  }
  bool solve(double &residual, double tolerance = 1e-6, int max_iter = 1000) {
    clear_error();
    ocu_pcg_params p = params();
    if (!check_ok(ocu_pcg_set_params(_s, &p))) return false;
    ocu_status st = ocu_pcg_solve(_s, &residual, tolerance, max_iter);
    if (st == OCU_ERR_NOT_CONVERGED) return false;
    return check_ok(st);
  }
  Grid3DDevice<T> &pressure() { return _pressure; }
  Grid3DDevice<T> &rhs() { return *rhs_grid; }
  Grid3DDevice<T> &coefficient() { return *coefficient_grid; }
};

typedef Sol_PCGPressure3DDevice<float> Sol_PCGPressure3DDeviceF;
typedef Sol_PCGPressure3DDevice<double> Sol_PCGPressure3DDeviceD;

// NetCDFGrid3DWriter / NetCDFGrid3DReader (gridnetcdf.h:67-183): the reference's grid files in the
// NetCDF classic format, without libnetcdf; the writer writes the file at close().
namespace detail {
template <typename T> struct nc_of;
template <> struct nc_of<float> { static const int value = OCU_NC_FLOAT; };
template <> struct nc_of<double> { static const int value = OCU_NC_DOUBLE; };
template <> struct nc_of<int> { static const int value = OCU_NC_INT; };
}  // namespace detail

class NetCDFGrid3DWriter {
  ocu_nc_writer *_w = nullptr;
  std::vector<float> _times;
 public:
  ~NetCDFGrid3DWriter() { if (_w) close(); }
  bool is_open() const { return _w != nullptr; }
  bool open(const char *filename, int nx, int ny, int nz, float hx = 1.0f, float hy = 1.0f, float hz = 1.0f) {
    return !_w && ocu_nc_writer_open(filename, nx, ny, nz, hx, hy, hz, &_w) == OCU_OK;
  }
  bool define_variable(const char *name, nc_type var_type, GridStaggering stag, float offsetx = 0.5f,
                       float offsety = 0.5f, float offsetz = 0.5f) {
    return ocu_nc_writer_define_variable(_w, name, var_type, stag, offsetx, offsety, offsetz) == OCU_OK;
  }
  bool add_time_level(float time, size_t &level) {
    int l = 0;
    if (ocu_nc_writer_add_time_level(_w, time, &l) != OCU_OK) return false;
    _times.push_back(time);
    level = (size_t)l;
    return true;
  }
  int get_time_level(float time) const {
    for (size_t i = 0; i < _times.size(); i++)
      if (_times[i] == time) return (int)i;
    return -1;
  }
  float get_time(int time_level) const { return _times[time_level]; }
  template <typename T>
  bool add_data(const char *name, const Grid3DHost<T> &grid, int time_level = 0) {
    if (time_level == 0 && _times.empty()) _times.push_back(0.0f);
    return ocu_nc_writer_add_data(_w, name, &grid.at(0, 0, 0), detail::nc_of<T>::value, grid.xstride(), grid.ystride(),
                                  grid.nx(), grid.ny(), grid.nz(), time_level) == OCU_OK;
  }
  bool close() {
    const bool ok = ocu_nc_writer_close(_w) == OCU_OK;
    _w = nullptr;
    _times.clear();
    return ok;
  }
};

class NetCDFGrid3DReader {
  ocu_nc_reader *_r = nullptr;
  int _nx = 0, _ny = 0, _nz = 0, _nt = 0;
  float _hx = 0, _hy = 0, _hz = 0;
  bool find(const char *name, int &t, int &x, int &y, int &z) const {
    int n = 0;
    ocu_nc_reader_num_variables(_r, &n);
    char buf[1024];
    for (int q = 0; q < n; q++)
      if (ocu_nc_reader_variable(_r, q, buf, (int)sizeof(buf), &t, &x, &y, &z) == OCU_OK && std::strcmp(buf, name) == 0)
        return true;
    return false;
  }
 public:
  ~NetCDFGrid3DReader() { close(); }
  bool is_open() const { return _r != nullptr; }
  bool open(const char *filename) {
    if (_r || ocu_nc_reader_open(filename, &_r) != OCU_OK) return false;
    return ocu_nc_reader_info(_r, &_nx, &_ny, &_nz, &_hx, &_hy, &_hz, &_nt) == OCU_OK;
  }
  int nx() const { return _nx; } int ny() const { return _ny; } int nz() const { return _nz; }
  float hx() const { return _hx; } float hy() const { return _hy; } float hz() const { return _hz; }
  int num_time_levels() const { return _nt; }
  float get_time(int time_level) const { float t = 0; ocu_nc_reader_get_time(_r, time_level, &t); return t; }
  std::vector<std::string> list_variables() const {
    std::vector<std::string> out;
    int n = 0;
    ocu_nc_reader_num_variables(_r, &n);
    char buf[1024];
    for (int q = 0; q < n; q++)
      if (ocu_nc_reader_variable(_r, q, buf, (int)sizeof(buf), nullptr, nullptr, nullptr, nullptr) == OCU_OK)
        out.push_back(buf);
    return out;
  }
  bool variable_type(const char *name, nc_type &type) const { int x, y, z; return find(name, type, x, y, z); }
  bool variable_size(const char *name, int &nx, int &ny, int &nz) const { int t; return find(name, t, nx, ny, nz); }
  template <typename T>
  bool read_variable(const char *name, Grid3DHost<T> &grid, int time_level = 0) const {
    return ocu_nc_reader_read(_r, name, &grid.at(0, 0, 0), detail::nc_of<T>::value, grid.xstride(), grid.ystride(),
                              grid.nx(), grid.ny(), grid.nz(), time_level) == OCU_OK;
  }
  bool close() {
    if (_r) ocu_nc_reader_close(_r);
    _r = nullptr;
    return true;
  }
};

}  // namespace ocu

#endif  // OCU_OPENCURRENT_H
