// Multigrid solver classes behind the ocu_mg_* C entry points.
#pragma once

#include <array>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <vector>

#include "co_mg.h"
#include "ir_chequer.h"
#include "mg_fused.h"
#include "ocu_internal.h"

namespace ocub {

// relax order (sol_mgpressure3d.h: RO_RED_BLACK, RO_BLACK_RED, RO_SYMMETRIC)
enum { RO_RED_BLACK = 0, RO_BLACK_RED = 1, RO_SYMMETRIC = 2 };

int mg_num_levels(int nx, int ny, int nz);

// The single-CTA coarse tail covers the 4^3 level only by default: measured at 256^3, a V-cycle
// takes 0.558 ms (FP32) / 0.787 ms (FP64) with the tail at 64 cells against 0.581 / 0.810 ms at
// 512 cells -- one SM runs a phase of an 8^3 level slower than a separate launch does.
// (Ensembles run one tail CTA per member and use a larger tail.)
constexpr int kDefaultTailCells = 64;
// The two-colour TMA pass is off unless asked for: at 256^3 FP32 it takes 110 us per sweep
// against 124 us for the two colour launches, but it is instruction-bound, slower in FP64, and a
// whole solve is not faster with it yet.
constexpr int kDefaultSweepCells = 0;
double mg_optimal_omega(double fx, double fy, double fz);

// The virtual level operations of Sol_MultigridPressure3DBase (sol_mgpressure3d.h:76-80).
struct CoreOps {
  virtual ~CoreOps() {}
  virtual ocu_status relax(int level, int iterations, int order) = 0;
  virtual ocu_status clear_zero(int level) = 0;
  virtual ocu_status apply_bc(int level) = 0;
  virtual ocu_status restrict_residuals(int fine, int coarse, double *l2, double *linf) = 0;
  virtual ocu_status prolong(int coarse, int fine) = 0;
  virtual ocu_status relax_sweep(int level, int color) = 0;
  virtual ocu_grid *grid(char which, int level) = 0;
  virtual int levels() const = 0;
  // clear_zero + apply_boundary_conditions
  virtual ocu_status clear_level(int level) = 0;
  // restrict_residuals split at the host wait: enqueue, then finish_norms for the numbers
  virtual ocu_status enqueue_restrict_residuals(int fine, int coarse, bool want_l2, bool want_linf) = 0;
  virtual ocu_status clear_and_restrict(int fine, bool want_l2, bool want_linf) = 0;
  virtual ocu_status finish_norms(int fine, double *l2, double *linf) = 0;
  // levels tail_start()..L-1 of a V-cycle in one launch
  virtual int tail_start() const = 0;
  virtual ocu_status cycle_tail(int s, int nu1, int nu2, int coarse_iters, bool symmetric) = 0;
  // hierarchies spread over several streams: make the solver's stream wait for all of them
  // (join), and all of them wait for the solver's stream (fork: at the start of a stream capture,
  // so that their work joins the captured graph)
  virtual ocu_status join() { return OCU_OK; }
  virtual ocu_status fork() { return OCU_OK; }
  virtual void on_stream(cudaStream_t) {}
  virtual void on_params(const ocu_mg_params &) {}
};

// Level hierarchy of one precision (Sol_MultigridPressure3DDevice<T> storage).
template <typename T>
struct MGCore : CoreOps {
  int num_levels = 0;
  std::vector<double> h;
  std::vector<std::array<int, 3>> dim;
  double omega = 1, fx = 1, fy = 1, fz = 1;
  std::vector<ocu_layout> lay;
  std::vector<ocu_grid *> grids_u, grids_b, grids_r;  // u[0] = pressure, b[0] = caller rhs
  std::vector<void *> diag;                           // FP64 diagonal tables
  ocu_bc_set bc{};
  bool update_bc_between_colors = false;
  bool disable_relax_on_host = false;
  cudaStream_t stream = nullptr;
  void *red_scratch = nullptr;
  double *d_norms = nullptr;
  double *h_norms = nullptr;
  void *rows = nullptr;           // per-row norm partials of level 0 (l2 then linf)
  long long rows_stride = 0;
  bool fused = true;              // fused kernels (ghost writes, residual+restrict, tail)
  bool store_residuals = false;   // keep r_grid filled (reference kernels) for read_r
  int tail_cells = kDefaultTailCells;    // levels with at most this many cells run in the tail kernel
  int sweep_cells = kDefaultSweepCells;  // levels with at least this many cells use the two-colour pass
  // two-colour pass: per level a second u buffer (ping-pong) and the TMA maps of u, u2 and b
  std::vector<ocu_grid *> grids_u2;
  std::vector<SweepTmap> tm_u, tm_u2, tm_b;
  int *d_err = nullptr;           // set by kernels whose bounded waits gave up (inside d_norms)
  int wait_limit = 0;             // polls of such a wait before it gives up (0 = the default)

  ~MGCore();
  ocu_status clear_level(int level) override;
  bool emit_ok(int level) const;
  bool sweep2_ok(int level) const;
  ocu_status ensure_sweep_buffers();
  ocu_status relax_pairs(int level, int iterations, int order);
  ocu_status enqueue_restrict_residuals(int fine, int coarse, bool want_l2, bool want_linf) override;
  ocu_status clear_and_restrict(int fine, bool want_l2, bool want_linf) override;
  ocu_status finish_norms(int fine, double *l2, double *linf) override;
  int tail_start() const override;
  ocu_status cycle_tail(int s, int nu1, int nu2, int coarse_iters, bool symmetric) override;
  void fill_tail_params(TailParams<T> &P, int s, int nu1, int nu2, int coarse_iters, bool symmetric,
                        T *const *u_origin, T *const *b_origin) const;
  // level count, spacings, operator factors, omega and layouts (no allocation)
  ocu_status set_geometry(const ocu_bc_set &bc, bool disable_host, int nx, int ny, int nz, double hx, double hy,
                          double hz, const ocu_layout &L0);
  ocu_status init(const ocu_bc_set &bc, bool disable_host, int nx, int ny, int nz, double hx, double hy,
                  double hz, ocu_grid *rhs, ocu_grid *pressure, cudaStream_t s);
  ocu_bc_set bc_at_level(int level) const;
  RelaxParams relax_params(int level) const;
  double hx(int l) const { return h[l] / std::sqrt(fx); }
  double hy(int l) const { return h[l] / std::sqrt(fy); }
  double hz(int l) const { return h[l] / std::sqrt(fz); }
  T *u0(int l) { return origin<T>(grids_u[l]); }
  T *b0(int l) { return origin<T>(grids_b[l]); }
  T *r0(int l) { return origin<T>(grids_r[l]); }

  ocu_status relax(int level, int iterations, int order) override;
  ocu_status clear_zero(int level) override;
  ocu_status apply_bc(int level) override;
  ocu_status restrict_residuals(int fine, int coarse, double *l2, double *linf) override;
  ocu_status prolong(int coarse, int fine) override;
  ocu_status relax_sweep(int level, int color) override {
    const T *dg = diag.empty() ? nullptr : (const T *)diag[level];
    return launch_relax_color<T>(u0(level), b0(level), lay[level], dg, color, relax_params(level), stream);
  }
  int levels() const override { return num_levels; }
  ocu_grid *grid(char which, int level) override {
    return which == 'u' ? grids_u[level] : which == 'b' ? grids_b[level] : which == 'r' ? grids_r[level] : nullptr;
  }
};

struct MGSolver {
  ocu_mg_kind kind;
  ocu_mg_params prm;
  MGCore<float> cf;
  MGCore<double> cd;
  bool double_mode = false;
  bool initialized = false;
  int num_levels = 0;
  ocu_grid *pressure = nullptr;   // u0 of the interface precision
  ocu_grid *rhs_f = nullptr;      // FP32 rhs of the mixed solvers
  struct GridDeleter {
    void operator()(ocu_grid *g) const {
      if (g) { cudaFree(g->buf); delete g; }
    }
  };
  std::unique_ptr<ocu_grid, GridDeleter> pressure_f;  // FP32 u0 of the mixed solvers
  std::unique_ptr<ChequerMG> chq;  // split-layout FP32 correction solver (OCU_MG_MIXED_IR)
  // multi-image solver (Sol_MultigridPressure3DDeviceCo): images, their devices, the cutoff
  // (grid_size_for_cutoff) and, once initialized, the hierarchy that replaces cf / cd
  int co_images = 0;
  std::vector<int> co_devices;
  long long co_cutoff_cells = 64LL * 64 * 64;
  std::unique_ptr<CoOps> co;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;  // used when the caller's stream is the legacy NULL stream
  ocu_mg_stats stats{};
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
  };
  std::map<std::pair<const void *, int>, GraphEntry> graphs;
  bool use_graphs = true;

  // OCU_B200_GRAPHS=0 in the environment replays nothing (every launch issued by the host)
  explicit MGSolver(ocu_mg_kind k, const ocu_mg_params &p) : kind(k), prm(p) {
    const char *g = std::getenv("OCU_B200_GRAPHS");
    use_graphs = !(g && g[0] == '0');
  }
  ~MGSolver();
  void clear_graphs();
  template <typename F> ocu_status run_segment(const void *core, int seg, F &&enqueue);
  ocu_status enq_down(CoreOps *c, int a, int b);
  ocu_status enq_tail_up(CoreOps *c, int s, int f);
  ocu_status do_fmg_graph(double tol, int max_iter, double *l2, double *linf);
  ocu_status do_vcycle_graph(double tol, int max_iter, double *l2, double *linf);

  CoreOps *active();
  int coarse_iters() const;
  ocu_status initialize_storage(int nx, int ny, int nz, double hx, double hy, double hz, ocu_grid *rhs);
  ocu_status initialize_storage_co(int nx_local, int ny, int nz, double hx, double hy, double hz,
                                   ocu_grid *const *rhs);
  ocu_status set_params(const ocu_mg_params &p);
  ocu_status apply_knobs();
  void set_stream(cudaStream_t s);
  ocu_status do_fmg(double tol, int max_iter, double *l2, double *linf);
  ocu_status do_vcycle(double tol, int max_iter, double *l2, double *linf);
  ocu_status cycle(CoreOps *c, int fine_level, double tol, double *l2, double *linf, bool *converged);
  ocu_status ir_residual(double *l2, double *linf);
  ocu_status mixed_warmstart_fmg(double tol, int max_iter, double *l2, double *linf);
  ocu_status ir_solve(double tol, int max_outer, double *l2, double *linf);
  ocu_status ir_solve_chequer(double tol, int max_outer, double *l2, double *linf);
  ocu_status ir_chequer_residual_tail();
  ocu_status fmg_dispatch(double tol, int max_iter, double *l2, double *linf);
  ocu_status solve(double *residual, double tol, int max_iter);
  ocu_status run_vcycles(int count);
  ocu_status run_fmg(int count);
  ocu_grid *level_grid(char which, int level);
};

}  // namespace ocub

struct ocu_mg {
  ocub::MGSolver s;
  ocu_mg(ocu_mg_kind k, const ocu_mg_params &p) : s(k, p) {}
};
