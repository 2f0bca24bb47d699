// Multi-image multigrid: Sol_MultigridPressure3DDeviceCo<T> (sol_mgpressure3d.h:184-242,
// sol_mgpressure3dco.cu:39-529).
//
// The reference runs one host thread per image (one GPU each) and meets at barriers that copy
// halo planes through pinned host memory.  Here one host thread drives every image in lockstep:
// an image owns a stream on its device and a slab hierarchy (levels above the cutoff, x extent
// divided by the image count); after each ghost refresh the x halo planes are copied device to
// device into the receiving image's ghost planes on the receiver's stream, after an event of the
// sender, and each sender's stream waits for its readers' copies before it next writes.  No kernel
// waits on another; all ordering is stream order and events, so N images may share one device.
//
// Kernels go without programmatic dependent launch here: between two kernels of an image's
// stream there are copies and event waits, which must complete before the next kernel starts.
//
// Per-cell work is the single-image kernels' on the slab layouts with the slab's own face rules
// (BC_NONE on a face whose ghost plane is a neighbour's copy), so when every slab's x extent is
// even above the cutoff the colour parity is the global one and the result after a fixed number
// of cycles is bit-identical to the single-image solver on the whole grid.  Norms are the images'
// reductions folded in image order in T (ThreadManager::barrier_reduce, thread.h:90-103).
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "co_mg.h"
#include "mg_solver.h"

namespace ocub {

namespace {

struct DevGuard {
  int prev = -1;
  DevGuard() { cudaGetDevice(&prev); }
  ~DevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

#define CO_CK(call, what) OCU_TRY(check_cuda((call), what))

ocu_grid *co_alloc(ocu_dtype dt, const ocu_layout &L, ocu_status *st) {
  ocu_grid *g = new ocu_grid;
  g->dtype = dt;
  g->L = L;
  g->owned = true;
  g->buf = nullptr;
  cudaError_t e = cudaMalloc(&g->buf, dtype_size(dt) * L.allocated);
  if (e == cudaSuccess) e = cudaMemset(g->buf, 0, dtype_size(dt) * L.allocated);
  if (e != cudaSuccess) {
    if (g->buf) cudaFree(g->buf);
    delete g;
    *st = check_cuda(e, "cudaMalloc (multi-image levels)");
    return nullptr;
  }
  return g;
}

void co_free(ocu_grid *g) {
  if (g) {
    cudaFree(g->buf);
    delete g;
  }
}

// First element of the memory block of x-plane x (x = -1 and x = nx are the ghost planes): the
// block runs over every y and z entry of the plane, ghosts and padding included, xstride long.
template <typename T>
T *plane(ocu_grid *g, int x) {
  return origin<T>(g) + (long long)x * g->L.xstride - (long long)g->L.gy * g->L.ystride - g->L.gz;
}

template <typename T>
struct CoMG : CoOps, CoreOps {
  struct Image {
    int dev = 0, neg = -1, pos = -1;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    MGCore<T> slab;  // levels 0 .. cutoff-1 of this image's slab
    ocu_grid *u_prolong = nullptr, *b_restrict = nullptr;  // the cutoff level over this slab
    ocu_grid *pressure = nullptr;
    bool own_pressure = false;
  };

  ocu_dtype dt = OCU_F32;
  int N = 0, L = 0, cutoff = 0;
  std::vector<std::array<int, 3>> gdim;
  std::vector<std::unique_ptr<Image>> im;
  MGCore<T> top;  // image 0: levels cutoff .. L-1 of the whole grid (top level t = level cutoff + t)
  int cdim[3] = {0, 0, 0};

  ~CoMG() override {
    DevGuard g;
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      if (m->stream) cudaStreamSynchronize(m->stream);
    }
    if (!top.grids_u.empty()) {
      co_free(top.grids_u[0]);  // level 0 of `top` is allocated here, not by MGCore
      co_free(top.grids_b[0]);
      top.grids_u[0] = top.grids_b[0] = nullptr;
    }
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      co_free(m->u_prolong);
      co_free(m->b_restrict);
      if (m->own_pressure) co_free(m->pressure);
      if (m->ev_a) cudaEventDestroy(m->ev_a);
      if (m->ev_b) cudaEventDestroy(m->ev_b);
      if (m->own_stream && m->stream) cudaStreamDestroy(m->stream);
    }
  }

  // ---- CoOps ----
  CoreOps *ops() override { return this; }
  ocu_grid *pressure(int image) override { return image >= 0 && image < N ? im[image]->pressure : nullptr; }
  int images() const override { return N; }
  int cutoff_level() const override { return cutoff; }
  const int *coarse_dim() const override { return cdim; }

  bool sliced(int level) const { return level < cutoff; }
  Image &zero() { return *im[0]; }

  // Fused kernels (ghost writes inside the colour sweep and the prolongation, residual and
  // restriction in one pass, the single-CTA coarse tail on image 0's levels); off with the
  // unfused parameter.  All of them give the same bits as the separate kernels.
  bool fused = true;

  // Ghost writes can ride in a slab's kernels when each BC_NONE face of the slab is one whose
  // ghost plane the halo copy then overwrites whole (a neighbour's face), and no periodic axis
  // of the slab is odd (the single-image rule).
  bool slab_emit(int level) const {
    if (!fused) return false;
    for (auto &m : im) {
      const ocu_bc_set b = m->slab.bc_at_level(level);
      if (b.ypos.type == OCU_BC_NONE || b.yneg.type == OCU_BC_NONE || b.zpos.type == OCU_BC_NONE ||
          b.zneg.type == OCU_BC_NONE)
        return false;
      if ((b.xneg.type == OCU_BC_NONE && m->neg < 0) || (b.xpos.type == OCU_BC_NONE && m->pos < 0)) return false;
      if (b.xneg.type == OCU_BC_PERIODIC || b.xpos.type == OCU_BC_PERIODIC) return false;
      const auto &d = m->slab.dim[level];
      if ((b.ypos.type == OCU_BC_PERIODIC || b.yneg.type == OCU_BC_PERIODIC) && (d[1] & 1)) return false;
      if ((b.zpos.type == OCU_BC_PERIODIC || b.zneg.type == OCU_BC_PERIODIC) && (d[2] & 1)) return false;
    }
    return true;
  }

  // ---- halo exchange (CoArrayManager::barrier_exchange of the u planes,
  //      sol_mgpressure3dco.cu:44-58, 440-470) ----
  ocu_status exchange(int level) {
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      CO_CK(cudaEventRecord(m->ev_a, m->stream), "cudaEventRecord (halo)");
    }
    const size_t bytes = (size_t)im[0]->slab.lay[level].xstride * sizeof(T);
    for (int i = 0; i < N; i++) {
      Image &m = *im[i];
      cudaSetDevice(m.dev);
      ocu_grid *g = m.slab.grids_u[level];
      const int nx = m.slab.dim[level][0];
      if (m.neg >= 0) {
        Image &q = *im[m.neg];
        if (m.neg != i) CO_CK(cudaStreamWaitEvent(m.stream, q.ev_a, 0), "cudaStreamWaitEvent (halo)");
        CO_CK(cudaMemcpyAsync(plane<T>(g, -1), plane<T>(q.slab.grids_u[level], nx - 1), bytes, cudaMemcpyDefault,
                              m.stream),
              "halo copy (x-)");
      }
      if (m.pos >= 0) {
        Image &p = *im[m.pos];
        if (m.pos != i) CO_CK(cudaStreamWaitEvent(m.stream, p.ev_a, 0), "cudaStreamWaitEvent (halo)");
        CO_CK(cudaMemcpyAsync(plane<T>(g, nx), plane<T>(p.slab.grids_u[level], 0), bytes, cudaMemcpyDefault,
                              m.stream),
              "halo copy (x+)");
      }
    }
    // a sender writes its edge planes again only after the images that read them have copied
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      CO_CK(cudaEventRecord(m->ev_b, m->stream), "cudaEventRecord (halo)");
    }
    for (int i = 0; i < N; i++) {
      Image &m = *im[i];
      cudaSetDevice(m.dev);
      if (m.neg >= 0 && m.neg != i) CO_CK(cudaStreamWaitEvent(m.stream, im[m.neg]->ev_b, 0), "cudaStreamWaitEvent");
      if (m.pos >= 0 && m.pos != i && m.pos != m.neg)
        CO_CK(cudaStreamWaitEvent(m.stream, im[m.pos]->ev_b, 0), "cudaStreamWaitEvent");
    }
    return OCU_OK;
  }

  // every image's stream waits for image 0's work so far, and image 0's for every image's
  ocu_status fence_with_zero() {
    Image &z = zero();
    cudaSetDevice(z.dev);
    CO_CK(cudaEventRecord(z.ev_a, z.stream), "cudaEventRecord");
    for (int i = 1; i < N; i++) {
      Image &m = *im[i];
      cudaSetDevice(m.dev);
      CO_CK(cudaStreamWaitEvent(m.stream, z.ev_a, 0), "cudaStreamWaitEvent");
    }
    return OCU_OK;
  }
  ocu_status zero_waits_all() {
    for (int i = 1; i < N; i++) {
      Image &m = *im[i];
      cudaSetDevice(m.dev);
      CO_CK(cudaEventRecord(m.ev_b, m.stream), "cudaEventRecord");
    }
    Image &z = zero();
    cudaSetDevice(z.dev);
    for (int i = 1; i < N; i++) CO_CK(cudaStreamWaitEvent(z.stream, im[i]->ev_b, 0), "cudaStreamWaitEvent");
    return OCU_OK;
  }

  // restricted right-hand sides of the slabs into image 0's cutoff level (the gather_b exchange,
  // sol_mgpressure3dco.cu:497-503)
  ocu_status gather_b() {
    Image &z = zero();
    for (int i = 0; i < N; i++) {
      Image &m = *im[i];
      cudaSetDevice(m.dev);
      CO_CK(cudaEventRecord(m.ev_a, m.stream), "cudaEventRecord (gather)");
    }
    cudaSetDevice(z.dev);
    const int slice = im[0]->b_restrict->L.nx;
    const size_t bytes = (size_t)slice * top.lay[0].xstride * sizeof(T);
    for (int i = 0; i < N; i++) {
      if (i) CO_CK(cudaStreamWaitEvent(z.stream, im[i]->ev_a, 0), "cudaStreamWaitEvent (gather)");
      CO_CK(cudaMemcpyAsync(plane<T>(top.grids_b[0], slice * i), plane<T>(im[i]->b_restrict, 0), bytes,
                            cudaMemcpyDefault, z.stream),
            "gather copy");
    }
    // an image restricts into its b_restrict again only after image 0 has copied it
    return fence_with_zero();
  }

  // image 0's cutoff-level u, one plane beyond each side, into every slab's u_prolong (the
  // scatter_u exchange, sol_mgpressure3dco.cu:505-510)
  ocu_status scatter_u() {
    OCU_TRY(fence_with_zero());
    const int slice = im[0]->u_prolong->L.nx;
    const size_t bytes = (size_t)(slice + 2) * top.lay[0].xstride * sizeof(T);
    for (int i = 0; i < N; i++) {
      Image &m = *im[i];
      cudaSetDevice(m.dev);
      CO_CK(cudaMemcpyAsync(plane<T>(m.u_prolong, -1), plane<T>(top.grids_u[0], slice * i - 1), bytes,
                            cudaMemcpyDefault, m.stream),
            "scatter copy");
    }
    // image 0 writes its cutoff level again only after every image has copied from it
    return zero_waits_all();
  }

  // ---- CoreOps ----
  int levels() const override { return L; }
  int tail_start() const override { return fused ? cutoff + top.tail_start() : L - 1; }

  ocu_grid *grid(char which, int level) override {
    if (level < 0 || level >= L) return nullptr;
    if (sliced(level)) return zero().slab.grid(which, level);
    return top.grid(which, level - cutoff);
  }

  // apply_boundary_conditions (sol_mgpressure3dco.cu:36-66)
  ocu_status apply_bc(int level) override {
    DevGuard g;
    PdlSuppress np_;
    if (!sliced(level)) {
      cudaSetDevice(zero().dev);
      return top.apply_bc(level - cutoff);
    }
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      OCU_TRY(m->slab.apply_bc(level));
    }
    return exchange(level);
  }

  ocu_status sweep_all(int level, int color) {
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      MGCore<T> &s = m->slab;
      const T *dg = s.diag.empty() ? nullptr : (const T *)s.diag[level];
      OCU_TRY(launch_relax_color<T>(s.u0(level), s.b0(level), s.lay[level], dg, color, s.relax_params(level),
                                    m->stream));
    }
    return OCU_OK;
  }

  // relax (sol_mgpressure3dco.cu:102-110 over sol_mgpressure3ddev.cu:190-248 with the ghosts
  // refreshed after every colour)
  ocu_status relax(int level, int iterations, int order) override {
    DevGuard g;
    PdlSuppress np_;
    // On the fused path every operation leaves the ghosts current, so the refresh the
    // reference makes first would rewrite the same values.
    if (!sliced(level)) {
      cudaSetDevice(zero().dev);
      if (!fused) OCU_TRY(top.apply_bc(level - cutoff));
      return top.relax(level - cutoff, iterations, order);
    }
    const bool emit = slab_emit(level);
    if (!emit) OCU_TRY(apply_bc(level));
    if (order == RO_SYMMETRIC) {
      if (iterations % 2 == 1) iterations++;
      if (iterations < 4) iterations = 4;
    }
    for (int it = 0; it < iterations; it++)
      for (int rb = 0; rb < 2; rb++) {
        int color = rb;
        if (order == RO_BLACK_RED || (order == RO_SYMMETRIC && it >= iterations / 2)) color = !rb;
        if (emit) {
          for (auto &m : im) {
            cudaSetDevice(m->dev);
            MGCore<T> &q = m->slab;
            const T *dg = q.diag.empty() ? nullptr : (const T *)q.diag[level];
            OCU_TRY(launch_relax_color_emit<T>(q.u0(level), q.b0(level), q.lay[level], dg, color, q.relax_params(level),
                                               q.hx(level), q.hy(level), q.hz(level), m->stream));
          }
          OCU_TRY(exchange(level));
        } else {
          OCU_TRY(sweep_all(level, color));
          OCU_TRY(apply_bc(level));
        }
      }
    return OCU_OK;
  }

  ocu_status relax_sweep(int level, int color) override {
    DevGuard g;
    PdlSuppress np_;
    if (!sliced(level)) {
      cudaSetDevice(zero().dev);
      return top.relax_sweep(level - cutoff, color);
    }
    OCU_TRY(sweep_all(level, color & 1));
    return exchange(level);
  }

  // clear_zero (sol_mgpressure3dco.cu:203-210)
  ocu_status clear_zero(int level) override {
    DevGuard g;
    PdlSuppress np_;
    if (!sliced(level)) {
      cudaSetDevice(zero().dev);
      return top.clear_zero(level - cutoff);
    }
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      OCU_TRY(m->slab.clear_zero(level));
    }
    return OCU_OK;
  }

  // Below level 0 the faces are homogeneous: the ghost rules map the cleared interior to +0,
  // the bits the clear wrote, so only level 0 refreshes its ghosts.
  ocu_status clear_level(int level) override {
    OCU_TRY(clear_zero(level));
    return level == 0 ? apply_bc(0) : OCU_OK;
  }

  // restrict_residuals (sol_mgpressure3dco.cu:112-178)
  int norm_mode = 0;  // 0: none pending, 1: images, 2: image 0's whole levels
  ocu_status enqueue_restrict_residuals(int fine, int coarse, bool want_l2, bool want_linf) override {
    return restrict_images(fine, coarse, want_l2, want_linf, false);
  }

  // zero_coarse: clear the coarse level's u too (in the restriction kernel when fused)
  ocu_status restrict_images(int fine, int coarse, bool want_l2, bool want_linf, bool zero_coarse) {
    DevGuard g;
    PdlSuppress np_;
    const bool do_restrict = fine != coarse;
    const bool norms = want_l2 || want_linf;
    if ((!do_restrict && coarse == cutoff) || fine >= cutoff) {
      cudaSetDevice(zero().dev);
      norm_mode = norms ? 2 : 0;
      if (zero_coarse) return top.clear_and_restrict(fine - cutoff, want_l2, want_linf);
      return top.enqueue_restrict_residuals(fine - cutoff, coarse - cutoff, want_l2, want_linf);
    }
    norm_mode = norms ? 1 : 0;
    if (zero_coarse && (coarse == cutoff || !fused)) OCU_TRY(clear_zero(coarse));
    if (fused) {
      for (auto &m : im) {
        cudaSetDevice(m->dev);
        MGCore<T> &q = m->slab;
        T *rows2 = want_l2 ? (T *)q.rows : nullptr;
        T *rowsinf = want_linf ? (T *)q.rows + q.rows_stride : nullptr;
        if (do_restrict) {
          const bool to_cut = coarse == cutoff;
          T *zu = (zero_coarse && !to_cut) ? static_cast<T *>(q.grids_u[coarse]->buf) : nullptr;
          const long long zn = zu ? q.lay[coarse].allocated : 0;
          OCU_TRY(launch_residual_restrict<T>(q.u0(fine), q.b0(fine), q.lay[fine],
                                              to_cut ? origin<T>(m->b_restrict) : q.b0(coarse),
                                              to_cut ? m->b_restrict->L : q.lay[coarse], q.h[fine], q.fx, q.fy, q.fz,
                                              rows2, rowsinf, m->stream, zu, zn));
        } else if (norms) {
          OCU_TRY(launch_residual_rows<T>(q.u0(fine), q.b0(fine), nullptr, nullptr, q.lay[fine], q.h[fine], q.fx, q.fy,
                                          q.fz, rows2, rowsinf, m->stream));
        }
        const long long nrows = (long long)q.dim[fine][0] * q.dim[fine][1];
        if (want_l2) OCU_TRY(launch_fold_rows<T>(rows2, nrows, false, q.red_scratch, q.d_norms, m->stream));
        if (want_linf) OCU_TRY(launch_fold_rows<T>(rowsinf, nrows, true, q.red_scratch, q.d_norms + 1, m->stream));
        if (norms)
          OCU_TRY(launch_readback(q.d_norms, q.h_norms, 2, m->stream));
      }
      if (do_restrict && coarse == cutoff) OCU_TRY(gather_b());
      return OCU_OK;
    }
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      MGCore<T> &s = m->slab;
      OCU_TRY(launch_residual<T>(s.u0(fine), s.b0(fine), s.r0(fine), s.lay[fine], s.h[fine], s.fx, s.fy, s.fz,
                                 m->stream));
      if (do_restrict) {
        if (coarse == cutoff)
          OCU_TRY(launch_restrict<T>(s.r0(fine), s.lay[fine], origin<T>(m->b_restrict), m->b_restrict->L, m->stream));
        else
          OCU_TRY(launch_restrict<T>(s.r0(fine), s.lay[fine], s.b0(coarse), s.lay[coarse], m->stream));
      }
      if (want_l2) OCU_TRY(launch_reduce<T>(s.r0(fine), s.lay[fine], OCU_REDUCE_SQRSUM, s.red_scratch, s.d_norms, m->stream));
      if (want_linf)
        OCU_TRY(launch_reduce<T>(s.r0(fine), s.lay[fine], OCU_REDUCE_MAXABS, s.red_scratch, s.d_norms + 1, m->stream));
      if (norms)
        OCU_TRY(launch_readback(s.d_norms, s.h_norms, 2, m->stream));
    }
    if (do_restrict && coarse == cutoff) OCU_TRY(gather_b());
    return OCU_OK;
  }

  ocu_status finish_norms(int fine, double *l2, double *linf) override {
    DevGuard g;
    PdlSuppress np_;
    if (norm_mode == 2 || !sliced(fine)) {
      cudaSetDevice(zero().dev);
      return top.finish_norms(fine - cutoff, l2, linf);
    }
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      CO_CK(cudaStreamSynchronize(m->stream), "norm readback");
    }
    // co_reduce_sqrsum / co_reduce_maxabs: each image's T result, folded in image order
    if (l2) {
      T rn = (T)im[0]->slab.h_norms[0];
      for (int i = 1; i < N; i++) rn = (T)im[i]->slab.h_norms[0] + rn;
      const auto &d = im[0]->slab.dim[fine];
      rn /= (T)((long long)d[0] * d[1] * d[2] * N);
      *l2 = (double)std::sqrt(rn);
    }
    if (linf) {
      T mx = (T)std::fabs((T)im[0]->slab.h_norms[1]);
      for (int i = 1; i < N; i++) {
        const T v = (T)std::fabs((T)im[i]->slab.h_norms[1]);
        mx = v > mx ? v : mx;
      }
      *linf = (double)mx;
    }
    return OCU_OK;
  }

  ocu_status restrict_residuals(int fine, int coarse, double *l2, double *linf) override {
    OCU_TRY(enqueue_restrict_residuals(fine, coarse, l2 != nullptr, linf != nullptr));
    if (l2 || linf) return finish_norms(fine, l2, linf);
    return OCU_OK;
  }

  // clear_level(fine + 1) then the restriction into it (level fine + 1 >= 1: no ghost refresh)
  ocu_status clear_and_restrict(int fine, bool want_l2, bool want_linf) override {
    return restrict_images(fine, fine + 1, want_l2, want_linf, true);
  }

  // prolong (sol_mgpressure3dco.cu:180-201)
  ocu_status prolong(int coarse, int fine) override {
    DevGuard g;
    PdlSuppress np_;
    if (coarse > cutoff) {
      cudaSetDevice(zero().dev);
      return top.prolong(coarse - cutoff, fine - cutoff);
    }
    if (coarse == cutoff) OCU_TRY(scatter_u());
    const bool emit = slab_emit(fine);
    for (auto &m : im) {
      cudaSetDevice(m->dev);
      MGCore<T> &s = m->slab;
      const T *uc = coarse == cutoff ? origin<T>(m->u_prolong) : s.u0(coarse);
      const ocu_layout &Lc = coarse == cutoff ? m->u_prolong->L : s.lay[coarse];
      if (emit)
        OCU_TRY(launch_prolong_emit<T>(uc, Lc, s.u0(fine), s.lay[fine], s.bc_at_level(fine), s.hx(fine), s.hy(fine),
                                       s.hz(fine), m->stream));
      else
        OCU_TRY(launch_prolong<T>(uc, Lc, s.u0(fine), s.lay[fine], m->stream));
    }
    return emit ? exchange(fine) : apply_bc(fine);
  }

  // the levels from s down, all on image 0 (s >= cutoff): its tail kernel or coarse relax
  ocu_status cycle_tail(int s, int nu1, int nu2, int coarse_iters, bool symmetric) override {
    DevGuard g;
    PdlSuppress np_;
    cudaSetDevice(zero().dev);
    return top.cycle_tail(s - cutoff, nu1, nu2, coarse_iters, symmetric);
  }

  ocu_status join() override {
    DevGuard g;
    PdlSuppress np_;
    return zero_waits_all();
  }

  ocu_status fork() override {
    DevGuard g;
    return fence_with_zero();
  }

  void on_stream(cudaStream_t s) override {
    zero().stream = s;
    zero().slab.stream = s;
    top.stream = s;
  }

  void on_params(const ocu_mg_params &p) override {
    top.disable_relax_on_host = p.disable_relax_on_host != 0;
    fused = top.fused = p.unfused == 0;
    top.tail_cells = p.tail_cells == 0 ? kDefaultTailCells : (p.tail_cells < 0 ? 0 : p.tail_cells);
  }
};

// Geometry of levels [first, last) of the global hierarchy G into core C, x extent divided by
// div; storage of level 0 of C supplied by the caller (u0, b0), the rest allocated here.
template <typename T>
ocu_status co_fill_core(MGCore<T> &C, const MGCore<T> &G, int first, int last, int div, const ocu_bc_set &bc,
                        ocu_grid *u0, ocu_grid *b0, const ocu_layout &L0, bool disable_host, bool fused,
                        int tail_cells, cudaStream_t s) {
  const ocu_dtype dt = sizeof(T) == 8 ? OCU_F64 : OCU_F32;
  const int n = last - first;
  C.stream = s;
  C.bc = bc;
  C.disable_relax_on_host = disable_host;
  C.update_bc_between_colors = true;  // sol_mgpressure3dco.cu:290
  C.fused = fused;
  C.tail_cells = tail_cells;
  C.num_levels = n;
  C.fx = G.fx; C.fy = G.fy; C.fz = G.fz;
  C.omega = G.omega;
  C.h.assign(G.h.begin() + first, G.h.begin() + last);
  C.dim.resize(n);
  C.lay.resize(n);
  for (int l = 0; l < n; l++) {
    C.dim[l] = {G.dim[first + l][0] / div, G.dim[first + l][1], G.dim[first + l][2]};
    if (l == 0) C.lay[0] = L0;
    else layout_compute(C.dim[l][0], C.dim[l][1], C.dim[l][2], 1, 1, 1, 0, 0, 0, &C.lay[l]);
  }
  C.grids_u.assign(n, nullptr);
  C.grids_b.assign(n, nullptr);
  C.grids_r.assign(n, nullptr);
  C.grids_u[0] = u0;
  C.grids_b[0] = b0;
  ocu_status st = OCU_OK;
  for (int l = 0; l < n; l++) {
    if (l > 0) {
      C.grids_u[l] = co_alloc(dt, C.lay[l], &st);
      if (!C.grids_u[l]) return st;
      C.grids_b[l] = co_alloc(dt, C.lay[l], &st);
      if (!C.grids_b[l]) return st;
    }
    C.grids_r[l] = co_alloc(dt, C.lay[l], &st);
    if (!C.grids_r[l]) return st;
  }
  if (sizeof(T) == 8) {
    C.diag.assign(n, nullptr);
    for (int l = 0; l < n; l++) {
      OCU_TRY(check_cuda(cudaMalloc(&C.diag[l], sizeof(T) * (size_t)C.dim[l][0] * C.dim[l][1]), "cudaMalloc(diag)"));
      OCU_TRY(launch_init_diag<T>((T *)C.diag[l], C.dim[l][0], C.dim[l][1], C.relax_params(l), s));
    }
  }
  const size_t rs = reduce_scratch_bytes(C.lay[0], sizeof(T));
  OCU_TRY(check_cuda(cudaMalloc(&C.red_scratch, rs), "cudaMalloc(reduce)"));
  OCU_TRY(check_cuda(cudaMemset(C.red_scratch, 0, rs), "cudaMemset(reduce)"));
  C.rows_stride = ((long long)C.dim[0][0] * C.dim[0][1] + 63) / 64 * 64;
  OCU_TRY(check_cuda(cudaMalloc(&C.rows, 2 * sizeof(T) * C.rows_stride), "cudaMalloc(norm rows)"));
  OCU_TRY(check_cuda(cudaMalloc(&C.d_norms, 4 * sizeof(double)), "cudaMalloc(norms)"));
  OCU_TRY(check_cuda(cudaMemset(C.d_norms, 0, 4 * sizeof(double)), "cudaMemset(norms)"));
  OCU_TRY(check_cuda(cudaMallocHost(&C.h_norms, 4 * sizeof(double)), "cudaMallocHost(norms)"));
  std::memset(C.h_norms, 0, 4 * sizeof(double));
  C.d_err = reinterpret_cast<int *>(C.d_norms + 2);
  return OCU_OK;
}

template <typename T>
ocu_status co_build(int N, const int *devices, int nxl, int ny, int nz, double hx, double hy, double hz,
                    ocu_grid *const *rhs, ocu_grid *pressure0, const ocu_mg_params &prm, long long cutoff_cells,
                    cudaStream_t stream0, std::unique_ptr<CoOps> *out) {
  const ocu_dtype dt = sizeof(T) == 8 ? OCU_F64 : OCU_F32;
  DevGuard guard;
  std::unique_ptr<CoMG<T>> c(new CoMG<T>());
  c->dt = dt;
  c->N = N;
  c->fused = prm.unfused == 0;
  const int tail_cells = prm.tail_cells == 0 ? kDefaultTailCells : (prm.tail_cells < 0 ? 0 : prm.tail_cells);
  MGCore<T> G;  // the global geometry (no storage)
  OCU_TRY(G.set_geometry(prm.bc, prm.disable_relax_on_host != 0, nxl * N, ny, nz, hx, hy, hz, rhs[0]->L));
  ocu_mgco_plan plan0;
  OCU_TRY(mgco_plan(nxl, ny, nz, N, 0, cutoff_cells, prm.bc, &plan0));
  c->L = G.num_levels;
  c->cutoff = plan0.cutoff_level;
  c->gdim = G.dim;
  if (c->cutoff >= c->L)
    return fail(OCU_ERR_UNSUPPORTED, "[ERROR] Sol_MultigridPressure3DDeviceCo::initialize_storage - no level of at most %lld cells: the coarsest level would be split across images", cutoff_cells);
  for (int l = 0; l < c->cutoff; l++)
    if (G.dim[l][0] % N)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_MultigridPressure3DDeviceCo::initialize_storage - level %d (%d cells along x) does not split across %d images", l, G.dim[l][0], N);
  for (int d = 0; d < 3; d++) c->cdim[d] = G.dim[c->L - 1][d];
  // peer access between the images' devices (NVLink); images on one device need none
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      if (devices[i] == devices[j]) continue;
      int can = 0;
      cudaDeviceCanAccessPeer(&can, devices[i], devices[j]);
      if (!can) continue;
      cudaSetDevice(devices[i]);
      const cudaError_t e = cudaDeviceEnablePeerAccess(devices[j], 0);
      if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
      else if (e != cudaSuccess) return check_cuda(e, "cudaDeviceEnablePeerAccess");
    }
  ocu_layout Lc;
  const int slice_c = G.dim[c->cutoff][0] / N;
  layout_compute(slice_c, G.dim[c->cutoff][1], G.dim[c->cutoff][2], 1, 1, 1, 0, 0, 0, &Lc);
  ocu_status st = OCU_OK;
  for (int i = 0; i < N; i++) {
    c->im.emplace_back(new typename CoMG<T>::Image());
    auto &m = *c->im.back();
    m.dev = devices[i];
    cudaSetDevice(m.dev);
    ocu_mgco_plan p;
    OCU_TRY(mgco_plan(nxl, ny, nz, N, i, cutoff_cells, prm.bc, &p));
    m.neg = p.neg_image;
    m.pos = p.pos_image;
    if (i == 0) {
      m.stream = stream0;
    } else {
      CO_CK(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking), "cudaStreamCreate");
      m.own_stream = true;
    }
    CO_CK(cudaEventCreateWithFlags(&m.ev_a, cudaEventDisableTiming), "cudaEventCreate");
    CO_CK(cudaEventCreateWithFlags(&m.ev_b, cudaEventDisableTiming), "cudaEventCreate");
    if (i == 0) {
      m.pressure = pressure0;
    } else {
      m.pressure = co_alloc(dt, rhs[i]->L, &st);
      if (!m.pressure) return st;
      m.own_pressure = true;
    }
    OCU_TRY(co_fill_core<T>(m.slab, G, 0, c->cutoff, N, p.local_bc, m.pressure, rhs[i], rhs[i]->L,
                            true, c->fused, tail_cells, m.stream));
    m.u_prolong = co_alloc(dt, Lc, &st);
    if (!m.u_prolong) return st;
    m.b_restrict = co_alloc(dt, Lc, &st);
    if (!m.b_restrict) return st;
  }
  // image 0's whole levels: the global faces, homogeneous (the cutoff is at least level 1)
  {
    cudaSetDevice(devices[0]);
    ocu_bc_set hb = prm.bc;
    bc_make_homogeneous(&hb);
    ocu_layout Lt;
    layout_compute(G.dim[c->cutoff][0], G.dim[c->cutoff][1], G.dim[c->cutoff][2], 1, 1, 1, 0, 0, 0, &Lt);
    ocu_grid *u0 = co_alloc(dt, Lt, &st);
    if (!u0) return st;
    ocu_grid *b0 = co_alloc(dt, Lt, &st);
    if (!b0) {
      co_free(u0);
      return st;
    }
    c->top.grids_u.assign(1, u0);  // owned by CoMG from here on, whatever happens below
    c->top.grids_b.assign(1, b0);
    OCU_TRY(co_fill_core<T>(c->top, G, c->cutoff, c->L, 1, hb, u0, b0, Lt, prm.disable_relax_on_host != 0,
                            c->fused, tail_cells, stream0));
  }
  for (auto &m : c->im) {
    cudaSetDevice(m->dev);
    CO_CK(cudaStreamSynchronize(m->stream), "initialize_storage");
  }
  *out = std::move(c);
  return OCU_OK;
}

}  // namespace

ocu_status mgco_plan(int nx_local, int ny, int nz, int num_images, int image, long long cutoff_cells,
                     const ocu_bc_set &bc, ocu_mgco_plan *out) {
  if (!out) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] mgco plan - null output");
  if (num_images < 1 || image < 0 || image >= num_images || nx_local < 1 || ny < 1 || nz < 1 || cutoff_cells < 1)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] mgco plan - bad arguments (%d images, image %d, %dx%dx%d, cutoff %lld)",
                num_images, image, nx_local, ny, nz, cutoff_cells);
  std::memset(out, 0, sizeof(*out));
  const long long nxg = (long long)nx_local * num_images;
  if (nxg > (1 << 30)) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] mgco plan - grid too large");
  out->num_levels = mg_num_levels((int)nxg, ny, nz);
  // _multi_thread_cutoff_level (sol_mgpressure3dco.cu:262-275): the first level >= 1 of at most
  // cutoff_cells cells, else num_levels
  out->cutoff_level = out->num_levels;
  long long dx = nxg, dy = ny, dz = nz;
  for (int l = 1; l < out->num_levels; l++) {
    dx /= 2; dy /= 2; dz /= 2;
    if (dx * dy * dz <= cutoff_cells) {
      out->cutoff_level = l;
      break;
    }
  }
  // neighbours (sol_mgpressure3dco.cu:286-294)
  out->neg_image = (image - 1 + num_images) % num_images;
  out->pos_image = (image + 1) % num_images;
  if (image == 0 && bc.xneg.type != OCU_BC_PERIODIC) out->neg_image = -1;
  if (image == num_images - 1 && bc.xpos.type != OCU_BC_PERIODIC) out->pos_image = -1;
  // this image's faces (sol_mgpressure3dco.cu:420-435)
  out->local_bc = bc;
  if (out->neg_image != -1) out->local_bc.xneg.type = OCU_BC_NONE;
  if (out->pos_image != -1) out->local_bc.xpos.type = OCU_BC_NONE;
  return OCU_OK;
}

ocu_status mgco_create(ocu_dtype dt, int num_images, const int *devices, int nx_local, int ny, int nz, double hx,
                       double hy, double hz, ocu_grid *const *rhs, ocu_grid *pressure0, const ocu_mg_params &prm,
                       long long cutoff_cells, cudaStream_t stream0, std::unique_ptr<CoOps> *out) {
  if (dt == OCU_F64)
    return co_build<double>(num_images, devices, nx_local, ny, nz, hx, hy, hz, rhs, pressure0, prm, cutoff_cells,
                            stream0, out);
  return co_build<float>(num_images, devices, nx_local, ny, nz, hx, hy, hz, rhs, pressure0, prm, cutoff_cells,
                         stream0, out);
}

}  // namespace ocub

// ---- C ABI -----------------------------------------------------------------------------------
using namespace ocub;

extern "C" {

ocu_status ocu_mgco_plan_compute(int nx_local, int ny, int nz, int num_images, int image, long long cutoff_cells,
                                 const ocu_bc_set *bc, ocu_mgco_plan *out) {
  if (!bc) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mgco_plan_compute - null bc");
  return mgco_plan(nx_local, ny, nz, num_images, image, cutoff_cells, *bc, out);
}

ocu_status ocu_mgco_create(ocu_mg_kind kind, const ocu_mg_params *params, int num_images, const int *devices,
                           ocu_mg **out) {
  if (!out) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mgco_create - null output");
  *out = nullptr;
  if (kind != OCU_MG_F32 && kind != OCU_MG_F64)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mgco_create - kind must be OCU_MG_F32 or OCU_MG_F64");
  if (num_images < 1 || num_images > 1024)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mgco_create - bad image count %d", num_images);
  ocu_mg_params p;
  if (params) p = *params;
  else ocu_mg_params_default(&p);
  ocu_mg *mg = new (std::nothrow) ocu_mg(kind, p);
  if (!mg) return fail(OCU_ERR_ALLOC, "[ERROR] ocu_mgco_create - out of host memory");
  mg->s.co_images = num_images;
  mg->s.co_devices.assign(num_images, 0);
  if (devices)
    for (int i = 0; i < num_images; i++) mg->s.co_devices[i] = devices[i];
  *out = mg;
  return OCU_OK;
}

ocu_status ocu_mgco_set_cutoff_cells(ocu_mg *mg, long long cells) {
  if (!mg || mg->s.co_images < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mgco_set_cutoff_cells - not a multi-image solver");
  if (mg->s.initialized) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mgco_set_cutoff_cells - already initialized");
  if (cells < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mgco_set_cutoff_cells - bad cell count %lld", cells);
  mg->s.co_cutoff_cells = cells;
  return OCU_OK;
}

ocu_status ocu_mgco_initialize_storage(ocu_mg *mg, int nx_local, int ny, int nz, double hx, double hy, double hz,
                                       ocu_grid *const *rhs) {
  if (!mg || mg->s.co_images < 1)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mgco_initialize_storage - not a multi-image solver");
  return mg->s.initialize_storage_co(nx_local, ny, nz, hx, hy, hz, rhs);
}

ocu_grid *ocu_mgco_pressure(ocu_mg *mg, int image) {
  if (!mg || !mg->s.co) return nullptr;
  return mg->s.co->pressure(image);
}

int ocu_mgco_num_images(const ocu_mg *mg) { return mg ? mg->s.co_images : 0; }

int ocu_mgco_cutoff_level(const ocu_mg *mg) { return (mg && mg->s.co) ? mg->s.co->cutoff_level() : -1; }

}  // extern "C"
