// Differentiable advection + projection chain on a periodic MAC grid, with a hand-written
// adjoint and checkpointing.
//
// Forward step n (fixed dt): dphi = A(u_n, phi_n) (passive advection), du = S(u_n) (self
// advection), phi_{n+1} = phi_n + dt dphi, u*_{n+1} = u_n + dt du, u_{n+1} = P u*_{n+1} with P
// the projection of Sol_ProjectDivergence3DDevice (divergence, multigrid pressure solve,
// gradient subtraction; sol_project3ddev.cu:58-71).  Each projection's pressure solve starts from
// the previous step's pressure, as the reference's projection solver keeps its pressure between
// solves; the forward chain starts from a zero pressure, and every checkpoint stores the pressure
// with the state, so a recomputed step starts from the same guess and reproduces the stored one
// exactly.  The adjoint chain's projections likewise start from the previous adjoint projection
// (from zero at the start of the backward pass).
//
// Adjoint step, given the cotangents (Lu', Lphi') of (u_{n+1}, phi_{n+1}):
//   Lu*   = P^T Lu' = P Lu'          (on the periodic grid D^T = -G, so P = I - G (DG)^-1 D is
//                                    symmetric: the same projection solver is reused)
//   Lu_n  = Lu* + dt (dS/du)^T Lu* + dt (dA/du)^T Lphi'
//   Lphi_n = Lphi' + dt (dA/dphi)^T Lphi'
// with the advection transposes of kernels_adjoint.cu.  States are checkpointed every k steps
// in the forward pass; the backward pass recomputes one segment of k states at a time.
#include <array>
#include <memory>
#include <vector>

#include "flow_solvers.h"
#include "ocu_internal.h"

namespace ocub {

template <typename T>
ocu_status launch_adj_passive(const T *u, const T *v, const T *w, const T *phi, const T *L, T *lam_phi, T *lu, T *lv,
                              T *lw, const ocu_layout &Lc, double c, double hx, double hy, double hz, int interp,
                              cudaStream_t s);
template <typename T>
ocu_status launch_adj_self(const T *u, const T *v, const T *w, const T *Lu, const T *Lv, const T *Lw, T *lu, T *lv,
                           T *lw, const ocu_layout &Lc, double c, double hx, double hy, double hz, int interp,
                           cudaStream_t s);

// Zero every element outside the nx x ny x nz block of cells/faces [0,n) (ghosts, padding).
template <typename T>
__global__ void k_zero_outside(T *buf, long long allocated, long long shift, long long xs, long long ys, int nx,
                               int ny, int nz) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= allocated) return;
  const long long r = q - shift;  // r = i*xs + j*ys + k for interior cells
  long long i = r >= 0 ? r / xs : -1;
  const long long rem = r - i * xs;
  const long long j = rem / ys, k = rem - j * ys;
  const bool inside = r >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz;
  if (!inside) buf[q] = (T)0;
}

struct AdjChain {
  ocu_dtype dtype = OCU_F32;
  int nx = 0, ny = 0, nz = 0, steps = 0, every = 1, interp = OCU_IT_FIRST_ORDER_UPWIND;
  double hx = 0, hy = 0, hz = 0, dt = 0, tol = 0;
  ocu_bc_set bc{};
  cudaStream_t stream = nullptr;
  using State = std::array<ocu_grid *, 4>;  // u, v, w, phi
  State W{}, D{}, Lam{}, Pl{}, nphi{};       // work state, derivatives, cotangents, projected, spare
  std::vector<State> ckpt, seg;
  std::vector<ocu_grid *> ckpt_p;  // the forward projection's pressure at each checkpoint
  std::unique_ptr<ProjectSolver> proj, proj_adj;
  bool have_forward = false;

  ~AdjChain() {
    if (stream) cudaStreamSynchronize(stream);
    proj.reset();
    proj_adj.reset();
    auto drop = [](State &s) {
      for (ocu_grid *g : s)
        if (g) { cudaFree(g->buf); delete g; }
    };
    drop(W); drop(D); drop(Lam); drop(Pl); drop(nphi);
    for (auto &s : ckpt) drop(s);
    for (auto &s : seg) drop(s);
    for (ocu_grid *g : ckpt_p)
      if (g) { cudaFree(g->buf); delete g; }
  }

  ocu_status make(const char which, ocu_grid **out) {
    ocu_layout L;
    OCU_TRY(ns_init_layout(nx, ny, nz, which, &L));
    ocu_grid *g = new ocu_grid{dtype, L, nullptr, true};
    cudaError_t e = cudaMalloc(&g->buf, dtype_size(dtype) * L.allocated);
    if (e != cudaSuccess) { delete g; return check_cuda(e, "cudaMalloc(adjoint chain)"); }
    *out = g;
    return check_cuda(cudaMemset(g->buf, 0, dtype_size(dtype) * L.allocated), "cudaMemset");
  }
  ocu_status make_state(State *s) {
    OCU_TRY(make('u', &(*s)[0]));
    OCU_TRY(make('v', &(*s)[1]));
    OCU_TRY(make('w', &(*s)[2]));
    return make('t', &(*s)[3]);
  }

  ocu_status init() {
    for (ocu_bc *f : {&bc.xpos, &bc.xneg, &bc.ypos, &bc.yneg, &bc.zpos, &bc.zneg}) {
      f->type = OCU_BC_PERIODIC;
      f->value = 0;
      f->aux_value = 0;
    }
    OCU_TRY(make_state(&W));
    OCU_TRY(make_state(&D));
    OCU_TRY(make_state(&Lam));
    OCU_TRY(make_state(&Pl));
    OCU_TRY(make_state(&nphi));
    ckpt.resize((steps + every - 1) / every);
    for (auto &s : ckpt) OCU_TRY(make_state(&s));
    seg.resize(every);
    for (auto &s : seg) OCU_TRY(make_state(&s));
    proj.reset(new ProjectSolver());
    proj->dtype = dtype;
    proj->set_stream(stream);
    OCU_TRY(proj->initialize_storage(nx, ny, nz, hx, hy, hz, W[0], W[1], W[2], bc));
    const ocu_layout &Lp = pressure(*proj)->L;
    ckpt_p.assign(ckpt.size(), nullptr);
    for (auto &g : ckpt_p) {
      g = new ocu_grid{dtype, Lp, nullptr, true};
      cudaError_t e = cudaMalloc(&g->buf, dtype_size(dtype) * Lp.allocated);
      if (e != cudaSuccess) {
        delete g;
        g = nullptr;
        return check_cuda(e, "cudaMalloc(adjoint chain checkpoint pressure)");
      }
    }
    proj_adj.reset(new ProjectSolver());
    proj_adj->dtype = dtype;
    proj_adj->set_stream(stream);
    return proj_adj->initialize_storage(nx, ny, nz, hx, hy, hz, Pl[0], Pl[1], Pl[2], bc);
  }

  void set_stream(cudaStream_t s) {
    stream = s;
    if (proj) proj->set_stream(s);
    if (proj_adj) proj_adj->set_stream(s);
  }

  ocu_status copy(ocu_grid *dst, const ocu_grid *src) {
    return check_cuda(cudaMemcpyAsync(dst->buf, src->buf, dtype_size(dtype) * dst->L.allocated,
                                      cudaMemcpyDeviceToDevice, stream), "adjoint chain copy");
  }
  ocu_status copy_state(State &dst, const State &src) {
    for (int c = 0; c < 4; c++) OCU_TRY(copy(dst[c], src[c]));
    return OCU_OK;
  }

  template <typename T> ocu_status ghosts(State &s) {
    OCU_TRY(launch_mac_bc_level1<T>(origin<T>(s[0]), origin<T>(s[1]), origin<T>(s[2]), s[0]->L, nx, ny, nz, bc,
                                    stream));
    return launch_bc_level1<T>(origin<T>(s[3]), s[3]->L, bc, hx, hy, hz, stream);
  }

  static ocu_grid *pressure(ProjectSolver &p) { return p.mg->s.pressure; }
  ocu_status clear_pressure(ProjectSolver &p) {
    return check_cuda(cudaMemsetAsync(pressure(p)->buf, 0, dtype_size(dtype) * pressure(p)->L.allocated, stream),
                      "clear pressure");
  }
  // the solve starts from the pressure the solver holds (the previous projection's)
  ocu_status project(ProjectSolver &p, double tolerance) {
    ocu_status st = p.solve(tolerance);
    return st == OCU_ERR_NOT_CONVERGED ? OCU_OK : st;
  }

  template <typename T> ocu_status step(State &s) {
    const ocu_layout &Lu = s[0]->L;
    OCU_TRY(launch_advect_passive<T>(origin<T>(s[0]), origin<T>(s[1]), origin<T>(s[2]), origin<T>(s[3]),
                                     origin<T>(D[3]), s[3]->L, nx, ny, nz, hx, hy, hz, interp, stream));
    OCU_TRY(launch_advect_self<T>(origin<T>(s[0]), origin<T>(s[1]), origin<T>(s[2]), origin<T>(D[0]),
                                  origin<T>(D[1]), origin<T>(D[2]), Lu, nx, ny, nz, hx, hy, hz, interp, stream));
    for (int c = 0; c < 4; c++) {
      T *x = (T *)s[c]->buf;
      OCU_TRY(launch_lincomb2<T>(x, s[c]->L, (T)1, x, (T)dt, (const T *)D[c]->buf, stream));
    }
    OCU_TRY(launch_bc_level1<T>(origin<T>(s[3]), s[3]->L, bc, hx, hy, hz, stream));
    // the projection solver is bound to W; other states go through W
    if (&s != &W) OCU_TRY(copy_state(W, s));
    OCU_TRY(project(*proj, tol));
    if (&s != &W) OCU_TRY(copy_state(s, W));
    return OCU_OK;
  }

  template <typename T> ocu_status forward(const State &in, ocu_grid *phi_out) {
    OCU_TRY(copy_state(W, in));
    OCU_TRY(ghosts<T>(W));
    OCU_TRY(clear_pressure(*proj));
    for (int n = 0; n < steps; n++) {
      if (n % every == 0) {
        OCU_TRY(copy_state(ckpt[n / every], W));
        OCU_TRY(copy(ckpt_p[n / every], pressure(*proj)));
      }
      OCU_TRY(step<T>(W));
    }
    OCU_TRY(copy(phi_out, W[3]));
    have_forward = true;
    return check_cuda(cudaStreamSynchronize(stream), "adjoint chain forward");
  }

  template <typename T> ocu_status adjoint_step(const State &s) {
    // Lu* = P Lu'
    for (int c = 0; c < 3; c++) OCU_TRY(copy(Pl[c], Lam[c]));
    OCU_TRY(project(*proj_adj, tol));
    // Lu_n = Lu* + dt (dS/du)^T Lu* + dt (dA/du)^T Lphi';  Lphi_n = Lphi' + dt (dA/dphi)^T Lphi'
    for (int c = 0; c < 3; c++) OCU_TRY(copy(Lam[c], Pl[c]));
    const ocu_layout &Lc = s[3]->L;
    OCU_TRY(launch_adj_self<T>(origin<T>(s[0]), origin<T>(s[1]), origin<T>(s[2]), origin<T>(Pl[0]), origin<T>(Pl[1]),
                               origin<T>(Pl[2]), origin<T>(Lam[0]), origin<T>(Lam[1]), origin<T>(Lam[2]), Lc, dt, hx,
                               hy, hz, interp, stream));
    OCU_TRY(launch_adj_passive<T>(origin<T>(s[0]), origin<T>(s[1]), origin<T>(s[2]), origin<T>(s[3]),
                                  origin<T>(Lam[3]), origin<T>(nphi[3]), origin<T>(Lam[0]), origin<T>(Lam[1]),
                                  origin<T>(Lam[2]), Lc, dt, hx, hy, hz, interp, stream));
    std::swap(Lam[3], nphi[3]);
    return OCU_OK;
  }

  template <typename T> ocu_status zero_outside(ocu_grid *g) {
    const ocu_layout &L = g->L;
    const unsigned blocks = (unsigned)((L.allocated + 255) / 256);
    k_zero_outside<T><<<blocks, 256, 0, stream>>>((T *)g->buf, L.allocated, L.shift, L.xstride, L.ystride, nx, ny,
                                                  nz);
    return check_launch("k_zero_outside");
  }

  template <typename T> ocu_status backward(const ocu_grid *lam_phi, State &out) {
    if (!have_forward) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] adjoint chain - backward before forward");
    for (int c = 0; c < 3; c++)
      OCU_TRY(check_cuda(cudaMemsetAsync(Lam[c]->buf, 0, dtype_size(dtype) * Lam[c]->L.allocated, stream), "clear"));
    OCU_TRY(copy(Lam[3], lam_phi));
    OCU_TRY(clear_pressure(*proj_adj));
    const int nseg = (int)ckpt.size();
    for (int sg = nseg - 1; sg >= 0; sg--) {
      const int n0 = sg * every, len = (steps - n0) < every ? steps - n0 : every;
      OCU_TRY(copy_state(W, ckpt[sg]));
      OCU_TRY(copy(pressure(*proj), ckpt_p[sg]));
      for (int j = 0; j < len; j++) {
        if (j > 0) OCU_TRY(step<T>(W));
        OCU_TRY(copy_state(seg[j], W));
      }
      for (int j = len - 1; j >= 0; j--) OCU_TRY(adjoint_step<T>(seg[j]));
    }
    for (int c = 0; c < 4; c++) {
      OCU_TRY(copy(out[c], Lam[c]));
      OCU_TRY(zero_outside<T>(out[c]));
    }
    return check_cuda(cudaStreamSynchronize(stream), "adjoint chain backward");
  }
};

}  // namespace ocub

// ---- C ABI ----------------------------------------------------------------------------------
struct ocu_adj {
  ocub::AdjChain c;
};

using namespace ocub;

static bool same_layout(const ocu_grid *g, const ocu_grid *ref) {
  return g && ref && g->dtype == ref->dtype && g->L.pnx == ref->L.pnx && g->L.pny == ref->L.pny &&
         g->L.pnz == ref->L.pnz && g->L.nx == ref->L.nx && g->L.ny == ref->L.ny && g->L.nz == ref->L.nz &&
         g->L.shift == ref->L.shift && g->L.allocated == ref->L.allocated;
}

extern "C" {

ocu_status ocu_adj_create(ocu_dtype dtype, int nx, int ny, int nz, double hx, double hy, double hz, int steps,
                          int checkpoint_every, double dt, int interp, double proj_tol, ocu_adj **out) {
  if (!out) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_create - null out");
  *out = nullptr;
  if (dtype != OCU_F32 && dtype != OCU_F64) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_create - bad dtype");
  if (nx < 4 || ny < 4 || nz < 4 || steps < 1 || checkpoint_every < 1)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_create - bad sizes, steps or checkpoint interval");
  if (!(hx > 0) || !(hy > 0) || !(hz > 0) || !(dt > 0) || !(proj_tol > 0))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_create - spacings, dt and tolerance must be positive");
  if (interp != OCU_IT_FIRST_ORDER_UPWIND && interp != OCU_IT_SECOND_ORDER_CENTERED)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_create - invalid interpolation type %d", interp);
  std::unique_ptr<ocu_adj> a(new ocu_adj());
  AdjChain &c = a->c;
  c.dtype = dtype;
  c.nx = nx; c.ny = ny; c.nz = nz;
  c.hx = hx; c.hy = hy; c.hz = hz;
  c.steps = steps;
  c.every = checkpoint_every;
  c.dt = dt;
  c.interp = interp;
  c.tol = proj_tol;
  OCU_TRY(c.init());
  *out = a.release();
  return OCU_OK;
}

void ocu_adj_destroy(ocu_adj *a) { delete a; }

ocu_status ocu_adj_set_stream(ocu_adj *a, ocu_stream s) {
  if (!a) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_set_stream - null handle");
  a->c.set_stream((cudaStream_t)s);
  return OCU_OK;
}

ocu_status ocu_adj_layout(const ocu_adj *a, char which, ocu_layout *layout) {
  if (!a || !layout) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_layout - null argument");
  return ns_init_layout(a->c.nx, a->c.ny, a->c.nz, which, layout);
}

ocu_status ocu_adj_forward(ocu_adj *a, const ocu_grid *u0, const ocu_grid *v0, const ocu_grid *w0,
                           const ocu_grid *phi0, ocu_grid *phi_out) {
  if (!a) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_forward - null handle");
  AdjChain &c = a->c;
  if (!same_layout(u0, c.W[0]) || !same_layout(v0, c.W[1]) || !same_layout(w0, c.W[2]) ||
      !same_layout(phi0, c.W[3]) || !same_layout(phi_out, c.W[3]))
    return fail(OCU_ERR_LAYOUT, "[ERROR] ocu_adj_forward - grids must have the chain's layouts (ocu_adj_layout)");
  AdjChain::State in{const_cast<ocu_grid *>(u0), const_cast<ocu_grid *>(v0), const_cast<ocu_grid *>(w0),
                     const_cast<ocu_grid *>(phi0)};
  return c.dtype == OCU_F64 ? c.forward<double>(in, phi_out) : c.forward<float>(in, phi_out);
}

ocu_status ocu_adj_backward(ocu_adj *a, const ocu_grid *lam_phi, ocu_grid *lam_u0, ocu_grid *lam_v0,
                            ocu_grid *lam_w0, ocu_grid *lam_phi0) {
  if (!a) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_adj_backward - null handle");
  AdjChain &c = a->c;
  if (!same_layout(lam_phi, c.W[3]) || !same_layout(lam_u0, c.W[0]) || !same_layout(lam_v0, c.W[1]) ||
      !same_layout(lam_w0, c.W[2]) || !same_layout(lam_phi0, c.W[3]))
    return fail(OCU_ERR_LAYOUT, "[ERROR] ocu_adj_backward - grids must have the chain's layouts (ocu_adj_layout)");
  AdjChain::State out{lam_u0, lam_v0, lam_w0, lam_phi0};
  return c.dtype == OCU_F64 ? c.backward<double>(lam_phi, out) : c.backward<float>(lam_phi, out);
}

ocu_status ocu_advect_passive_adjoint(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w,
                                      const ocu_grid *phi, const ocu_grid *lam_dphi, ocu_grid *lam_phi,
                                      ocu_grid *lam_u, ocu_grid *lam_v, ocu_grid *lam_w, int nx, int ny, int nz,
                                      double c, double hx, double hy, double hz, int interp, ocu_stream s) {
  const ocu_grid *all[] = {v, w, phi, lam_dphi, lam_phi, lam_u, lam_v, lam_w};
  if (!u) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] passive advection adjoint - null grid");
  for (const ocu_grid *g : all)
    if (!g || g->dtype != u->dtype || g->L.xstride != u->L.xstride || g->L.ystride != u->L.ystride ||
        g->L.shift != u->L.shift)
      return fail(OCU_ERR_LAYOUT, "[ERROR] passive advection adjoint - grids must share one padded layout");
  if (nx < 1 || ny < 1 || nz < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] passive advection adjoint - bad size");
  ocu_layout Lc = phi->L;
  Lc.nx = nx; Lc.ny = ny; Lc.nz = nz;
  if (u->dtype == OCU_F64)
    return launch_adj_passive<double>(origin<double>(u), origin<double>(v), origin<double>(w), origin<double>(phi),
                                      origin<double>(lam_dphi), origin<double>(lam_phi), origin<double>(lam_u),
                                      origin<double>(lam_v), origin<double>(lam_w), Lc, c, hx, hy, hz, interp,
                                      (cudaStream_t)s);
  return launch_adj_passive<float>(origin<float>(u), origin<float>(v), origin<float>(w), origin<float>(phi),
                                   origin<float>(lam_dphi), origin<float>(lam_phi), origin<float>(lam_u),
                                   origin<float>(lam_v), origin<float>(lam_w), Lc, c, hx, hy, hz, interp,
                                   (cudaStream_t)s);
}

ocu_status ocu_advect_self_adjoint(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w, const ocu_grid *lam_du,
                                   const ocu_grid *lam_dv, const ocu_grid *lam_dw, ocu_grid *lam_u, ocu_grid *lam_v,
                                   ocu_grid *lam_w, int nx, int ny, int nz, double c, double hx, double hy, double hz,
                                   int interp, ocu_stream s) {
  const ocu_grid *all[] = {v, w, lam_du, lam_dv, lam_dw, lam_u, lam_v, lam_w};
  if (!u) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] self advection adjoint - null grid");
  for (const ocu_grid *g : all)
    if (!g || g->dtype != u->dtype || g->L.xstride != u->L.xstride || g->L.ystride != u->L.ystride ||
        g->L.shift != u->L.shift)
      return fail(OCU_ERR_LAYOUT, "[ERROR] self advection adjoint - grids must share one padded layout");
  if (nx < 1 || ny < 1 || nz < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] self advection adjoint - bad size");
  ocu_layout Lc = u->L;
  Lc.nx = nx; Lc.ny = ny; Lc.nz = nz;
  if (u->dtype == OCU_F64)
    return launch_adj_self<double>(origin<double>(u), origin<double>(v), origin<double>(w), origin<double>(lam_du),
                                   origin<double>(lam_dv), origin<double>(lam_dw), origin<double>(lam_u),
                                   origin<double>(lam_v), origin<double>(lam_w), Lc, c, hx, hy, hz, interp,
                                   (cudaStream_t)s);
  return launch_adj_self<float>(origin<float>(u), origin<float>(v), origin<float>(w), origin<float>(lam_du),
                                origin<float>(lam_dv), origin<float>(lam_dw), origin<float>(lam_u),
                                origin<float>(lam_v), origin<float>(lam_w), Lc, c, hx, hy, hz, interp,
                                (cudaStream_t)s);
}

}  // extern "C"
