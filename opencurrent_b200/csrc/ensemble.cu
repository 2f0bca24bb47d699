// Ensembles of independent pressure solves (the batched form of
// Sol_MultigridPressure3DDevice<T>::solve, sol_mgpressure3d.cpp:332-370, over many right-hand
// sides of uneven sizes).
//
// Members are grouped into size classes (identical nx, ny, nz and spacings).  A class keeps one
// array per level holding every member's grid at a fixed member stride, so each step of the
// multigrid schedule is ONE launch over all members of the class (the batched kernels of
// kernels_mg_fused.cu), and the coarse end of a cycle is one CTA per member.  Convergence is
// decided on the device per member, with the host driver's arithmetic (l2 = sqrt(sum/N) in T,
// compared with the member's tolerance after the level-0 pre-smooth): a member that converged
// gets its final ghost fill and is skipped by every later launch.  Each class records three CUDA
// graphs -- INIT (ghost fill + initial norm), RAMP (restriction chain + FMG ramp) and CYCLE (one
// level-0 V-cycle with its convergence check) -- and replays CYCLE until no member is active;
// classes run concurrently on their own streams.  Each member's result is bit-identical to a
// single-grid solve of that member with the same parameters.
//
// Per class a small autotuner times the whole class solve for a few (nu1, nu2) smoothing pairs
// and colour-sweep block shapes and keeps the fastest (ocu_ens_autotune).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "mg_fused.h"
#include "mg_solver.h"
#include "ocu_internal.h"

namespace ocub {

__global__ void k_ens_reset(int *state, int *vcycles, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) {
    state[m] = 1;
    vcycles[m] = 0;
  }
}

struct EnsBase {
  virtual ~EnsBase() {}
  virtual ocu_status solve(const double *tol, int max_iter, int *converged) = 0;
  virtual ocu_status autotune(const double *tol, int max_iter) = 0;
  virtual ocu_status member_stats(int m, ocu_mg_stats *st) const = 0;
  virtual ocu_grid *rhs(int m) = 0;
  virtual ocu_grid *pressure(int m) = 0;
  virtual int classes() const = 0;
  virtual ocu_status class_info(int c, int dims[3], int *members, ocu_ens_tuning *t) const = 0;
  virtual ocu_status set_tuning(int c, const ocu_ens_tuning &t) = 0;
  virtual void set_stream(cudaStream_t s) = 0;
};

template <typename T>
struct EnsClass {
  MGCore<T> geo;                        // level geometry and coefficients (no grids of its own)
  int nx = 0, ny = 0, nz = 0, members = 0;
  std::vector<int> ids;                 // ensemble member index of each class member
  std::vector<long long> ms;            // member stride per level (elements)
  std::vector<T *> ubase, bbase;        // level arrays: members * ms[l]
  std::vector<T *> uo, bo;              // origin of member 0 per level
  T *rows = nullptr, *partial = nullptr;
  long long nrows = 0, pstride = 0;
  double *sums = nullptr, *tol = nullptr, *last_l2 = nullptr;
  int *state = nullptr, *vcycles = nullptr, *active = nullptr;
  int *h_active = nullptr;              // pinned copy of *active
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaGraphExec_t g_init = nullptr, g_ramp = nullptr, g_cycle = nullptr;
  int kernels_init = 0, kernels_ramp = 0, kernels_cycle = 0;
  ocu_ens_tuning tune{2, 2, {32, 4, 2}, 0.0};
  int ts = 0;                           // first level of the coarse tail

  ~EnsClass() {
    clear_graphs();
    for (T *p : ubase) cudaFree(p);
    for (T *p : bbase) cudaFree(p);
    cudaFree(rows);
    cudaFree(partial);
    cudaFree(sums);
    cudaFree(tol);
    cudaFree(last_l2);
    cudaFree(state);
    cudaFree(vcycles);
    cudaFree(active);
    if (h_active) cudaFreeHost(h_active);
    if (done) cudaEventDestroy(done);
    if (stream) cudaStreamDestroy(stream);
  }
  void clear_graphs() {
    if (g_init) cudaGraphExecDestroy(g_init);
    if (g_ramp) cudaGraphExecDestroy(g_ramp);
    if (g_cycle) cudaGraphExecDestroy(g_cycle);
    g_init = g_ramp = g_cycle = nullptr;
  }
  BatchSel sel(int want) const { return BatchSel{state, want}; }
  int levels() const { return geo.num_levels; }

  ocu_status relax(int l, int iterations, int order, int want) {
    const RelaxParams p = geo.relax_params(l);
    const T *dg = geo.diag.empty() ? nullptr : (const T *)geo.diag[l];
    if (order == RO_SYMMETRIC) {
      if (iterations % 2 == 1) iterations++;
      if (iterations < 4) iterations = 4;
    }
    for (int it = 0; it < iterations; it++)
      for (int rb = 0; rb < 2; rb++) {
        int color = rb;
        if (order == RO_BLACK_RED || (order == RO_SYMMETRIC && it >= iterations / 2)) color = !rb;
        OCU_TRY(launch_relax_color_emit_b<T>(uo[l], bo[l], geo.lay[l], dg, color, p, geo.hx(l), geo.hy(l),
                                             geo.hz(l), sel(want), ms[l], members, tune.relax_block, stream));
      }
    return OCU_OK;
  }
  ocu_status clear(int l) {  // clear_zero + homogeneous ghost fill of every member (all zeros)
    return check_cuda(cudaMemsetAsync(ubase[l], 0, sizeof(T) * ms[l] * members, stream), "ensemble clear");
  }
  ocu_status restrict_to(int f, bool norms) {
    return launch_residual_restrict_b<T>(uo[f], bo[f], geo.lay[f], bo[f + 1], geo.lay[f + 1], geo.h[f], geo.fx,
                                         geo.fy, geo.fz, norms ? rows : nullptr, sel(1), ms[f], ms[f + 1], members,
                                         stream);
  }
  ocu_status tail(int s, bool symmetric) {
    TailParams<T> P;
    geo.fill_tail_params(P, s, tune.nu1, tune.nu2, coarse_iters(), symmetric, uo.data(), bo.data());
    TailBatch tb;
    std::memset(&tb, 0, sizeof(tb));
    tb.sel = sel(1);
    for (int l = s; l < levels(); l++) tb.ms[l - s] = ms[l];
    return launch_coarse_tail_batch<T>(P, tb, members, stream);
  }
  int coarse_iters() const {
    const auto &d = geo.dim[levels() - 1];
    const int a = d[0] * d[1], b = d[1] * d[2], c = d[0] * d[2];
    return (a > b ? (a > c ? a : c) : (b > c ? b : c)) / 2;
  }
  ocu_status down(int a, int b) {
    for (int l = a; l < b; l++) {
      OCU_TRY(relax(l, tune.nu1, RO_RED_BLACK, 1));
      OCU_TRY(clear(l + 1));
      OCU_TRY(restrict_to(l, false));
    }
    return OCU_OK;
  }
  ocu_status tail_up(int s, int f, bool sym) {
    OCU_TRY(tail(s, sym));
    for (int l = s - 1; l >= f; l--) {
      OCU_TRY(launch_prolong_emit_b<T>(uo[l + 1], geo.lay[l + 1], uo[l], geo.lay[l], geo.bc_at_level(l), geo.hx(l),
                                       geo.hy(l), geo.hz(l), sel(1), ms[l + 1], ms[l], members, stream));
      if (l > 0) OCU_TRY(relax(l, tune.nu2, sym ? RO_BLACK_RED : RO_RED_BLACK, 1));
    }
    return OCU_OK;
  }
  ocu_status norms0() {
    return launch_fold_rows_b<T>(rows, nrows, partial, pstride, sums, sel(1), members, stream);
  }
};


template <typename T>
struct Ensemble : EnsBase {
  ocu_mg_params prm;
  int count = 0;
  int tail_cells = 4096;  // one CTA per member runs the coarse end: all SMs stay busy
  std::vector<std::unique_ptr<EnsClass<T>>> cls;
  std::vector<std::pair<int, int>> where;  // member -> (class, index in class)
  std::vector<ocu_grid> rhs_view, p_view;
  cudaStream_t user = nullptr;
  cudaEvent_t start_ev = nullptr;

  ~Ensemble() override {
    for (auto &c : cls)
      if (c->stream) cudaStreamSynchronize(c->stream);
    if (start_ev) cudaEventDestroy(start_ev);
  }

  ocu_status create(int n, const int *dims, const double *h, const ocu_mg_params &p) {
    prm = p;
    count = n;
    if (prm.convergence != OCU_CONVERGENCE_L2)
      return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ocu_ens_create - ensembles decide convergence on the L2 norm only");
    // group by (dims, spacings); larger classes first so they start first
    std::map<std::tuple<int, int, int, double, double, double>, int> key;
    std::vector<std::tuple<int, int, int, double, double, double>> keys;
    where.assign(n, {0, 0});
    std::vector<int> cls_of(n);
    for (int m = 0; m < n; m++) {
      auto k = std::make_tuple(dims[3 * m], dims[3 * m + 1], dims[3 * m + 2], h[3 * m], h[3 * m + 1], h[3 * m + 2]);
      auto it = key.find(k);
      if (it == key.end()) {
        it = key.emplace(k, (int)keys.size()).first;
        keys.push_back(k);
      }
      cls_of[m] = it->second;
    }
    std::vector<int> order(keys.size());
    for (size_t c = 0; c < keys.size(); c++) order[c] = (int)c;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
      const long long na = (long long)std::get<0>(keys[a]) * std::get<1>(keys[a]) * std::get<2>(keys[a]);
      const long long nb = (long long)std::get<0>(keys[b]) * std::get<1>(keys[b]) * std::get<2>(keys[b]);
      return na > nb;
    });
    std::vector<int> rank(keys.size());
    for (size_t r = 0; r < order.size(); r++) rank[order[r]] = (int)r;
    for (size_t r = 0; r < order.size(); r++) {
      cls.emplace_back(new EnsClass<T>());
      auto &c = *cls.back();
      std::tie(c.nx, c.ny, c.nz, std::ignore, std::ignore, std::ignore) = keys[order[r]];
    }
    for (int m = 0; m < n; m++) {
      auto &c = *cls[rank[cls_of[m]]];
      where[m] = {rank[cls_of[m]], (int)c.ids.size()};
      c.ids.push_back(m);
    }
    for (size_t r = 0; r < cls.size(); r++) {
      const auto &k = keys[order[r]];
      OCU_TRY(init_class(*cls[r], std::get<3>(k), std::get<4>(k), std::get<5>(k)));
    }
    rhs_view.resize(n);
    p_view.resize(n);
    for (int m = 0; m < n; m++) {
      auto &c = *cls[where[m].first];
      const int i = where[m].second;
      const ocu_dtype dt = sizeof(T) == 8 ? OCU_F64 : OCU_F32;
      rhs_view[m] = ocu_grid{dt, c.geo.lay[0], c.bbase[0] + i * c.ms[0], false};
      p_view[m] = ocu_grid{dt, c.geo.lay[0], c.ubase[0] + i * c.ms[0], false};
    }
    OCU_TRY(check_cuda(cudaEventCreateWithFlags(&start_ev, cudaEventDisableTiming), "cudaEventCreate"));
    return check_cuda(cudaDeviceSynchronize(), "ocu_ens_create");
  }

  ocu_status init_class(EnsClass<T> &c, double hx, double hy, double hz) {
    c.members = (int)c.ids.size();
    ocu_layout L0;
    layout_compute(c.nx, c.ny, c.nz, 1, 1, 1, 0, 0, 0, &L0);
    OCU_TRY(c.geo.set_geometry(prm.bc, prm.disable_relax_on_host != 0, c.nx, c.ny, c.nz, hx, hy, hz, L0));
    const int L = c.levels();
    if (L < 2)
      return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ocu_ens_create - grid (%d,%d,%d) has a single multigrid level",
                  c.nx, c.ny, c.nz);
    for (int l = 0; l < L; l++)
      if (!c.geo.emit_ok(l))
        return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ocu_ens_create - BC_NONE faces or odd periodic axes are not "
                                         "supported in ensembles");
    c.geo.tail_cells = tail_cells;
    c.ts = c.geo.tail_start();
    c.tune.nu1 = prm.nu1;
    c.tune.nu2 = prm.nu2;
    OCU_TRY(check_cuda(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "cudaStreamCreate"));
    OCU_TRY(check_cuda(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming), "cudaEventCreate"));
    c.geo.stream = c.stream;
    c.ms.resize(L);
    c.ubase.assign(L, nullptr);
    c.bbase.assign(L, nullptr);
    c.uo.resize(L);
    c.bo.resize(L);
    for (int l = 0; l < L; l++) {
      c.ms[l] = (c.geo.lay[l].allocated + 63) / 64 * 64;  // 256-byte aligned members
      const size_t bytes = sizeof(T) * (size_t)c.ms[l] * c.members;
      OCU_TRY(check_cuda(cudaMalloc(&c.ubase[l], bytes), "cudaMalloc(ensemble u)"));
      OCU_TRY(check_cuda(cudaMalloc(&c.bbase[l], bytes), "cudaMalloc(ensemble b)"));
      OCU_TRY(check_cuda(cudaMemset(c.ubase[l], 0, bytes), "cudaMemset"));
      OCU_TRY(check_cuda(cudaMemset(c.bbase[l], 0, bytes), "cudaMemset"));
      c.uo[l] = c.ubase[l] + c.geo.lay[l].shift;
      c.bo[l] = c.bbase[l] + c.geo.lay[l].shift;
    }
    if (sizeof(T) == 8) {
      c.geo.diag.assign(L, nullptr);
      for (int l = 0; l < L; l++) {
        OCU_TRY(check_cuda(cudaMalloc(&c.geo.diag[l], sizeof(T) * (size_t)c.geo.dim[l][0] * c.geo.dim[l][1]),
                           "cudaMalloc(diag)"));
        OCU_TRY(launch_init_diag<T>((T *)c.geo.diag[l], c.geo.dim[l][0], c.geo.dim[l][1], c.geo.relax_params(l),
                                    c.stream));
      }
    }
    c.nrows = (long long)c.nx * c.ny;
    c.pstride = (c.nrows + 255) / 256;
    OCU_TRY(check_cuda(cudaMalloc(&c.rows, sizeof(T) * c.nrows * c.members), "cudaMalloc(rows)"));
    OCU_TRY(check_cuda(cudaMalloc(&c.partial, sizeof(T) * c.pstride * c.members), "cudaMalloc(partial)"));
    OCU_TRY(check_cuda(cudaMalloc(&c.sums, sizeof(double) * c.members), "cudaMalloc(sums)"));
    OCU_TRY(check_cuda(cudaMalloc(&c.tol, sizeof(double) * c.members), "cudaMalloc(tol)"));
    OCU_TRY(check_cuda(cudaMalloc(&c.last_l2, sizeof(double) * c.members), "cudaMalloc(l2)"));
    OCU_TRY(check_cuda(cudaMalloc(&c.state, sizeof(int) * c.members), "cudaMalloc(state)"));
    OCU_TRY(check_cuda(cudaMalloc(&c.vcycles, sizeof(int) * c.members), "cudaMalloc(vcycles)"));
    OCU_TRY(check_cuda(cudaMalloc(&c.active, sizeof(int)), "cudaMalloc(active)"));
    OCU_TRY(check_cuda(cudaMallocHost(&c.h_active, sizeof(int)), "cudaMallocHost(active)"));
    OCU_TRY(check_cuda(cudaMemset(c.state, 0, sizeof(int) * c.members), "cudaMemset"));
    OCU_TRY(check_cuda(cudaMemset(c.vcycles, 0, sizeof(int) * c.members), "cudaMemset"));
    OCU_TRY(check_cuda(cudaMemset(c.last_l2, 0, sizeof(double) * c.members), "cudaMemset"));
    return OCU_OK;
  }

  // Stream-capture `enqueue` on the class stream into an executable graph.
  template <typename F>
  ocu_status capture(EnsClass<T> &c, cudaGraphExec_t *exec, int *kernels, F &&enqueue) {
    OCU_TRY(check_cuda(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture"));
    set_capturing(true);
    const unsigned long long n0 = launch_count_captured();
    ocu_status st;
    {
      PdlSuppress no_pdl;  // the classes run concurrently on their own streams
      st = enqueue();
    }
    *kernels = (int)(launch_count_captured() - n0);
    set_capturing(false);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c.stream, &g);
    if (st != OCU_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    OCU_TRY(check_cuda(e, "cudaStreamEndCapture"));
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    return check_cuda(e, "cudaGraphInstantiate");
  }

  // INIT, RAMP and CYCLE of one class (do_fmg, sol_mgpressure3d.cpp:113-251, per member).
  ocu_status build_graphs(EnsClass<T> &c) {
    if (c.g_cycle) return OCU_OK;
    const bool sym = prm.make_symmetric_operator != 0;
    const int L = c.levels();
    const ocu_layout &L0 = c.geo.lay[0];
    OCU_TRY(capture(c, &c.g_init, &c.kernels_init, [&]() -> ocu_status {
      k_ens_reset<<<(c.members + 255) / 256, 256, 0, c.stream>>>(c.state, c.vcycles, c.members);
      OCU_TRY(check_launch("k_ens_reset"));
      OCU_TRY(launch_bc_fill_b<T>(c.uo[0], L0, c.geo.bc_at_level(0), c.geo.hx(0), c.geo.hy(0), c.geo.hz(0),
                                  c.sel(1), c.ms[0], c.members, c.state, false, c.stream));
      OCU_TRY(launch_residual_rows_b<T>(c.uo[0], c.bo[0], L0, c.geo.h[0], c.geo.fx, c.geo.fy, c.geo.fz, c.rows,
                                        c.sel(1), c.ms[0], c.members, c.stream));
      OCU_TRY(c.norms0());
      OCU_TRY(launch_converge_b<T>(c.sums, (long long)c.nx * c.ny * c.nz, c.tol, c.state, c.vcycles, c.last_l2,
                                   c.active, c.members, true, c.stream));
      return check_cuda(cudaMemcpyAsync(c.h_active, c.active, sizeof(int), cudaMemcpyDeviceToHost, c.stream),
                        "active count");
    }));
    OCU_TRY(capture(c, &c.g_ramp, &c.kernels_ramp, [&]() -> ocu_status {
      for (int l = 0; l < L - 1; l++) {
        OCU_TRY(c.clear(l + 1));
        OCU_TRY(c.restrict_to(l, false));
      }
      for (int f = L - 1; f >= 1; f--) {
        const int s = c.ts > f ? c.ts : f;
        OCU_TRY(c.down(f, s));
        OCU_TRY(c.tail_up(s, f, sym));
        OCU_TRY(launch_prolong_emit_b<T>(c.uo[f], c.geo.lay[f], c.uo[f - 1], c.geo.lay[f - 1],
                                         c.geo.bc_at_level(f - 1), c.geo.hx(f - 1), c.geo.hy(f - 1),
                                         c.geo.hz(f - 1), c.sel(1), c.ms[f], c.ms[f - 1], c.members, c.stream));
      }
      return OCU_OK;
    }));
    OCU_TRY(capture(c, &c.g_cycle, &c.kernels_cycle, [&]() -> ocu_status {
      OCU_TRY(c.relax(0, c.tune.nu1, RO_RED_BLACK, 1));
      OCU_TRY(c.clear(1));
      OCU_TRY(c.restrict_to(0, true));
      OCU_TRY(c.norms0());
      OCU_TRY(launch_converge_b<T>(c.sums, (long long)c.nx * c.ny * c.nz, c.tol, c.state, c.vcycles, c.last_l2,
                                   c.active, c.members, false, c.stream));
      OCU_TRY(check_cuda(cudaMemcpyAsync(c.h_active, c.active, sizeof(int), cudaMemcpyDeviceToHost, c.stream),
                         "active count"));
      // members that converged in this cycle: final ghost fill, then retired
      OCU_TRY(launch_bc_fill_b<T>(c.uo[0], L0, c.geo.bc_at_level(0), c.geo.hx(0), c.geo.hy(0), c.geo.hz(0),
                                  c.sel(2), c.ms[0], c.members, c.state, true, c.stream));
      OCU_TRY(c.down(1, c.ts));
      return c.tail_up(c.ts, 0, sym);
    }));
    return OCU_OK;
  }

  ocu_status launch_graph(EnsClass<T> &c, cudaGraphExec_t g, int kernels) {
    OCU_TRY(check_cuda(cudaGraphLaunch(g, c.stream), "cudaGraphLaunch"));
    count_launch(kernels);
    return OCU_OK;
  }

  // Solve the given classes to their members' tolerances; returns the members converged.
  ocu_status run(const std::vector<int> &which, const double *tol, int max_iter, int *converged) {
    if (max_iter < 0) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_solve - negative max_iter %d", max_iter);
    OCU_TRY(check_cuda(cudaEventRecord(start_ev, user), "cudaEventRecord"));
    std::vector<int> live;
    for (int ci : which) {
      EnsClass<T> &c = *cls[ci];
      std::vector<double> t(c.members);
      for (int i = 0; i < c.members; i++) {
        t[i] = tol[c.ids[i]];
        if (!(t[i] >= 0))
          return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_solve - bad tolerance for member %d", c.ids[i]);
      }
      OCU_TRY(build_graphs(c));
      OCU_TRY(check_cuda(cudaStreamWaitEvent(c.stream, start_ev, 0), "cudaStreamWaitEvent"));
      OCU_TRY(check_cuda(cudaMemcpyAsync(c.tol, t.data(), sizeof(double) * c.members, cudaMemcpyHostToDevice,
                                         c.stream), "tolerances"));
      OCU_TRY(launch_graph(c, c.g_init, c.kernels_init));
      OCU_TRY(launch_graph(c, c.g_ramp, c.kernels_ramp));
      live.push_back(ci);
    }
    for (int cyc = 0; cyc <= max_iter && !live.empty(); cyc++) {
      for (int ci : live) OCU_TRY(launch_graph(*cls[ci], cls[ci]->g_cycle, cls[ci]->kernels_cycle));
      std::vector<int> next;
      for (int ci : live) {
        OCU_TRY(check_cuda(cudaStreamSynchronize(cls[ci]->stream), "ensemble cycle"));
        if (*cls[ci]->h_active > 0) next.push_back(ci);
      }
      live.swap(next);
    }
    for (int ci : which) OCU_TRY(check_cuda(cudaStreamSynchronize(cls[ci]->stream), "ensemble solve"));
    int conv = 0;
    for (int ci : which) {
      EnsClass<T> &c = *cls[ci];
      std::vector<int> st(c.members);
      OCU_TRY(check_cuda(cudaMemcpy(st.data(), c.state, sizeof(int) * c.members, cudaMemcpyDeviceToHost), "state"));
      for (int v : st) conv += v == 0;
    }
    if (converged) *converged = conv;
    return OCU_OK;
  }

  ocu_status solve(const double *tol, int max_iter, int *converged) override {
    std::vector<int> all(cls.size());
    for (size_t c = 0; c < cls.size(); c++) all[c] = (int)c;
    int conv = 0;
    OCU_TRY(run(all, tol, max_iter, &conv));
    if (converged) *converged = conv;
    if (conv < count) {
      set_error("[WARNING] ocu_ens_solve - %d of %d members did not reach their tolerance", count - conv, count);
      return OCU_ERR_NOT_CONVERGED;
    }
    return OCU_OK;
  }

  // Per class: time the whole class solve (zero initial guess) for every candidate smoothing
  // pair and colour-sweep block shape; keep the one that converges the most members, the
  // fastest among those; leave the pressures zeroed.
  ocu_status autotune(const double *tol, int max_iter) override {
    static const int nus[][2] = {{2, 2}, {1, 1}, {2, 1}, {3, 3}, {1, 2}};
    static const int blocks[][3] = {{32, 4, 2}, {32, 8, 1}, {16, 8, 2}, {32, 2, 4}};
    cudaEvent_t e0, e1;
    OCU_TRY(check_cuda(cudaEventCreate(&e0), "cudaEventCreate"));
    OCU_TRY(check_cuda(cudaEventCreate(&e1), "cudaEventCreate"));
    ocu_status result = OCU_OK;
    for (size_t ci = 0; ci < cls.size() && result == OCU_OK; ci++) {
      EnsClass<T> &c = *cls[ci];
      const ocu_ens_tuning original = c.tune;
      ocu_ens_tuning best = c.tune;
      best.ms = 1e300;
      int best_conv = -1;
      for (const auto &nu : nus) {
        for (const auto &bl : blocks) {
          ocu_ens_tuning t{nu[0], nu[1], {bl[0], bl[1], bl[2]}, 0.0};
          apply_tuning(c, t);
          for (int rep = 0; rep < 2 && result == OCU_OK; rep++) {  // first run records the graphs
            // (members that cannot reach their tolerance make run() report it; that is data here)
            result = check_cuda(cudaMemsetAsync(c.ubase[0], 0, sizeof(T) * c.ms[0] * c.members, c.stream), "clear");
            if (result != OCU_OK) break;
            result = check_cuda(cudaStreamSynchronize(c.stream), "sync");
            if (result != OCU_OK) break;
            int conv = 0;
            result = check_cuda(cudaEventRecord(e0, c.stream), "cudaEventRecord");
            if (result == OCU_OK) result = run({(int)ci}, tol, max_iter, &conv);
            if (result == OCU_OK) result = check_cuda(cudaEventRecord(e1, c.stream), "cudaEventRecord");
            if (result == OCU_OK) result = check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0;
            if (result == OCU_OK) result = check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            if (result == OCU_OK && rep == 1 && (conv > best_conv || (conv == best_conv && ms < best.ms))) {
              best = t;
              best.ms = ms;
              best_conv = conv;
            }
          }
        }
      }
      if (best_conv < 0) best = original;
      apply_tuning(c, best);
      if (result == OCU_OK)
        result = check_cuda(cudaMemsetAsync(c.ubase[0], 0, sizeof(T) * c.ms[0] * c.members, c.stream), "clear");
      if (result == OCU_OK) result = check_cuda(cudaStreamSynchronize(c.stream), "sync");
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return result;
  }

  void apply_tuning(EnsClass<T> &c, const ocu_ens_tuning &t) {
    const double ms = c.tune.ms;
    c.tune = t;
    if (t.ms == 0) c.tune.ms = ms;
    c.clear_graphs();
  }

  ocu_status member_stats(int m, ocu_mg_stats *st) const override {
    const EnsClass<T> &c = *cls[where[m].first];
    const int i = where[m].second;
    int vc = 0;
    double l2 = 0;
    OCU_TRY(check_cuda(cudaMemcpy(&vc, c.vcycles + i, sizeof(int), cudaMemcpyDeviceToHost), "stats"));
    OCU_TRY(check_cuda(cudaMemcpy(&l2, c.last_l2 + i, sizeof(double), cudaMemcpyDeviceToHost), "stats"));
    std::memset(st, 0, sizeof(*st));
    st->num_levels = c.levels();
    st->vcycles = vc;
    st->last_l2 = l2;
    st->omega = c.geo.omega;
    return OCU_OK;
  }
  ocu_grid *rhs(int m) override { return &rhs_view[m]; }
  ocu_grid *pressure(int m) override { return &p_view[m]; }
  int classes() const override { return (int)cls.size(); }
  ocu_status class_info(int ci, int dims[3], int *members, ocu_ens_tuning *t) const override {
    const EnsClass<T> &c = *cls[ci];
    if (dims) dims[0] = c.nx, dims[1] = c.ny, dims[2] = c.nz;
    if (members) *members = c.members;
    if (t) *t = c.tune;
    return OCU_OK;
  }
  ocu_status set_tuning(int ci, const ocu_ens_tuning &t) override {
    if (t.nu1 < 0 || t.nu2 < 0 || t.relax_block[0] < 1 || t.relax_block[1] < 1 || t.relax_block[2] < 1 ||
        t.relax_block[0] * t.relax_block[1] * t.relax_block[2] > 256)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_set_tuning - bad smoothing counts or block shape");
    apply_tuning(*cls[ci], t);
    return OCU_OK;
  }
  void set_stream(cudaStream_t s) override { user = s; }
};

}  // namespace ocub

// ---- C ABI ----------------------------------------------------------------------------------
struct ocu_ens {
  std::unique_ptr<ocub::EnsBase> impl;
  int count = 0;
};

using namespace ocub;

#define ENS_CHECK(e)                                                                         \
  do {                                                                                       \
    if (!(e) || !(e)->impl) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ensemble - null handle"); \
  } while (0)

extern "C" {

ocu_status ocu_ens_create(ocu_dtype dtype, int members, const int *dims, const double *h,
                          const ocu_mg_params *params, ocu_ens **out) {
  if (!out || !dims || !h) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_create - null argument");
  *out = nullptr;
  if (members < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_create - members must be >= 1");
  if (dtype != OCU_F32 && dtype != OCU_F64) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_create - bad dtype");
  for (int m = 0; m < members; m++) {
    if (dims[3 * m] < 2 || dims[3 * m + 1] < 2 || dims[3 * m + 2] < 2)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_create - member %d has bad dimensions", m);
    for (int a = 0; a < 3; a++)
      if (!(h[3 * m + a] > 0) || !std::isfinite(h[3 * m + a]))
        return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_create - member %d has a bad spacing", m);
  }
  ocu_mg_params p;
  if (params) p = *params; else ocu_mg_params_default(&p);
  std::unique_ptr<ocu_ens> e(new ocu_ens());
  e->count = members;
  ocu_status st;
  if (dtype == OCU_F32) {
    auto *impl = new Ensemble<float>();
    e->impl.reset(impl);
    st = impl->create(members, dims, h, p);
  } else {
    auto *impl = new Ensemble<double>();
    e->impl.reset(impl);
    st = impl->create(members, dims, h, p);
  }
  if (st != OCU_OK) return st;
  *out = e.release();
  return OCU_OK;
}

void ocu_ens_destroy(ocu_ens *e) { delete e; }

ocu_status ocu_ens_set_stream(ocu_ens *e, ocu_stream s) {
  ENS_CHECK(e);
  e->impl->set_stream((cudaStream_t)s);
  return OCU_OK;
}

ocu_status ocu_ens_rhs(ocu_ens *e, int member, ocu_grid **out) {
  ENS_CHECK(e);
  if (!out || member < 0 || member >= e->count) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_rhs - bad member");
  *out = e->impl->rhs(member);
  return OCU_OK;
}

ocu_status ocu_ens_pressure(ocu_ens *e, int member, ocu_grid **out) {
  ENS_CHECK(e);
  if (!out || member < 0 || member >= e->count)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_pressure - bad member");
  *out = e->impl->pressure(member);
  return OCU_OK;
}

ocu_status ocu_ens_solve(ocu_ens *e, const double *tol, int max_iter, int *converged) {
  ENS_CHECK(e);
  if (!tol) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_solve - null tolerances");
  return e->impl->solve(tol, max_iter, converged);
}

ocu_status ocu_ens_autotune(ocu_ens *e, const double *tol, int max_iter) {
  ENS_CHECK(e);
  if (!tol) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_autotune - null tolerances");
  return e->impl->autotune(tol, max_iter);
}

ocu_status ocu_ens_member_stats(const ocu_ens *e, int member, ocu_mg_stats *stats) {
  ENS_CHECK(e);
  if (!stats || member < 0 || member >= e->count)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_member_stats - bad member");
  return e->impl->member_stats(member, stats);
}

ocu_status ocu_ens_num_classes(const ocu_ens *e, int *n) {
  ENS_CHECK(e);
  if (!n) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_num_classes - null argument");
  *n = e->impl->classes();
  return OCU_OK;
}

ocu_status ocu_ens_class_info(const ocu_ens *e, int cls, int *dims, int *members, ocu_ens_tuning *tuning) {
  ENS_CHECK(e);
  if (cls < 0 || cls >= e->impl->classes())
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_class_info - bad class %d", cls);
  return e->impl->class_info(cls, dims, members, tuning);
}

ocu_status ocu_ens_set_tuning(ocu_ens *e, int cls, const ocu_ens_tuning *tuning) {
  ENS_CHECK(e);
  if (!tuning || cls < 0 || cls >= e->impl->classes())
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_ens_set_tuning - bad class %d", cls);
  return e->impl->set_tuning(cls, *tuning);
}

}  // extern "C"
