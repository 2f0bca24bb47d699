#include <cstdlib>
// Error reporting, layout arithmetic and BoundaryConditionSet helpers shared by the library.
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "ocu_internal.h"

namespace ocub {

static thread_local char g_last_error[512] = "";
static std::atomic<unsigned long long> g_launches{0};

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

ocu_status fail(ocu_status st, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return st;
}

ocu_status check_cuda(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return OCU_OK;
  set_error("[ERROR] %s - CUDA error \"%s\"", what, cudaGetErrorString(e));
  return OCU_ERR_CUDA;
}

bool pdl_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("OCU_B200_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

static thread_local bool g_pdl_suppressed = false;
bool pdl_suppressed() { return g_pdl_suppressed; }
void set_pdl_suppressed(bool on) { g_pdl_suppressed = on; }

ocu_status check_launch(const char *what) {
  count_launch();
  return check_cuda(cudaGetLastError(), what);
}

// Launches recorded while a stream capture is open do not run; they are counted separately and
// credited to the global count each time the captured graph is launched.
static thread_local bool g_capturing = false;
static thread_local unsigned long long g_captured = 0;

void count_launch(int n) {
  if (g_capturing) g_captured += (unsigned long long)n;
  else g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed);
}

unsigned long long launch_count() { return g_launches.load(); }

void set_capturing(bool on) { g_capturing = on; }

unsigned long long launch_count_captured() { return g_captured; }

const char *last_error_text() { return g_last_error; }

// Grid3DDevice<T>::init (ocustorage/grid3ddev.cu:358-400): pnz rounded up to 16, 16-gz
// elements of pre-padding so that k=0 of every row starts on a 16-element boundary.
void layout_compute(int nx, int ny, int nz, int gx, int gy, int gz, int padx, int pady, int padz,
                    ocu_layout *L) {
  std::memset(L, 0, sizeof(*L));
  const int pre_padding = 16 - gz;
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

BCDev to_dev(const ocu_bc_set &bc) {
  BCDev d;
  const ocu_bc *f[6] = {&bc.xpos, &bc.xneg, &bc.ypos, &bc.yneg, &bc.zpos, &bc.zneg};
  for (int i = 0; i < 6; i++) {
    d.type[i] = f[i]->type;
    d.value[i] = f[i]->value;
    d.aux[i] = f[i]->aux_value;
  }
  return d;
}

static bool face_in(const ocu_bc &b, int t1, int t2, int t3, int t4) {
  return b.type == t1 || b.type == t2 || b.type == t3 || b.type == t4;
}

bool bc_check_scalar(const ocu_bc_set &s) {
  const ocu_bc *f[6] = {&s.xpos, &s.xneg, &s.ypos, &s.yneg, &s.zpos, &s.zneg};
  for (int i = 0; i < 6; i++)
    if (!face_in(*f[i], OCU_BC_NONE, OCU_BC_PERIODIC, OCU_BC_DIRICHELET, OCU_BC_NEUMANN)) return false;
  return true;
}

bool bc_check_mac(const ocu_bc_set &s) {
  const ocu_bc *f[6] = {&s.xpos, &s.xneg, &s.ypos, &s.yneg, &s.zpos, &s.zneg};
  for (int i = 0; i < 6; i++)
    if (!face_in(*f[i], OCU_BC_NONE, OCU_BC_PERIODIC, OCU_BC_FORCED_INFLOW_VARIABLE_SLIP, -1))
      return false;
  return true;
}

bool bc_any_periodic(const ocu_bc_set &s) {
  return s.xpos.type == OCU_BC_PERIODIC || s.xneg.type == OCU_BC_PERIODIC ||
         s.ypos.type == OCU_BC_PERIODIC || s.yneg.type == OCU_BC_PERIODIC ||
         s.zpos.type == OCU_BC_PERIODIC || s.zneg.type == OCU_BC_PERIODIC;
}

// BoundaryConditionSet::make_homogeneous (ocuutil/boundary_condition.h:88-101)
void bc_make_homogeneous(ocu_bc_set *s) {
  ocu_bc *f[6] = {&s->xpos, &s->xneg, &s->ypos, &s->yneg, &s->zpos, &s->zneg};
  for (int i = 0; i < 6; i++) f[i]->value = f[i]->aux_value = 0;
}

// Sol_MultigridPressure3DBase::bc_diag_mod (ocuequation/sol_mgpressure3d.cpp:49-64)
double bc_diag_mod(const ocu_bc &b, double factor) {
  if (b.type == OCU_BC_DIRICHELET) return factor;
  if (b.type == OCU_BC_NEUMANN) return -factor;
  return 0;
}

// check_float takes a float (ocuutil/float_routines.h:33-51).
bool check_float(float f) { return std::isfinite(f); }

}  // namespace ocub
