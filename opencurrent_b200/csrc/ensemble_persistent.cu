// Persistent refinement ensembles: many independent pressure solves of uneven sizes in ONE
// kernel launch.  No reference counterpart as a whole; each member is the solve contract of
// Sol_MultigridPressure3DBase::solve (sol_mgpressure3d.cpp:332-370: the residual's L2 norm
// sqrt(sum r^2 / N) against an absolute tolerance, a bounded number of cycles) run as an FP64
// iterative refinement whose corrections are FP32 multigrid solves on the red/black split layout
// (the library's own inner solver, chq_device.cuh).
//
// Schedule.  The launch is persistent: as many blocks as fit on the GPU at once, each taking
// the next member from a device counter (members ordered largest first) and running that
// member's whole solve before taking another -- FP64 ghost fill, FP64 residual and its norm,
// and while the norm is above the member's tolerance an FP32 correction (the right-hand side
// restricted to the coarse levels, the small levels solved inside the block's shared memory,
// nested iteration back up, `cycles` V-cycles at level 0) added to the FP64 pressure.  Phases
// of a member are separated by block barriers only: no block ever waits for another block, so
// the launch has no inter-block spin waits to bound.  The FP32 levels live in a per-block
// scratch hierarchy sized for the largest member; the FP64 right-hand sides and pressures are
// the members' own grids (standard layout, ghost 1).  A solve is the counter reset plus this
// launch, captured once as a CUDA graph and replayed.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "bc_device.cuh"
#include "chq_device.cuh"
#include "mg_solver.h"
#include "ocu_internal.h"

namespace ocub {

using namespace chq;

namespace {

constexpr int kPensMaxLevels = 12;

// One FP32 level of a member: geometry, the float offset of its four colour arrays (u0, u1, b0,
// b1) in the block's scratch hierarchy, its coarse-pair count and operator coefficients.
struct PensLevel {
  int nx, ny, nz, rz;
  int ysh, zsh;  // log2 of ny, nz when powers of two, else -1 (the shared-memory tail)
  FDiv fq, fy;   // division by rz/4 and by ny
  FDiv fcm;      // pairs per row of this level (as the coarse level of a transfer)
  long long off;
  ChqK k;
};

struct PensOuter {
  double fxh, fyh, fzh, dg;
};

struct PensMember {
  double *x;          // origin of the FP64 pressure (cell (0, 0, 0))
  const double *b;    // origin of the FP64 right-hand side
  long long xs, ys;
  int nx, ny, nz, M;  // M = pairs per row at level 0
  FDiv fM, fY;        // division by M and by ny
  int nlev, ts;       // FP32 levels; first level of the shared-memory tail
  int vec;            // FP64 rows allow 16-byte pairs
  int pad_;
  double inv_n;       // 1 / (nx ny nz)
  double hx, hy, hz;  // ghost-rule spacings
  PensOuter oc;
  BCDev bcd;          // the member's boundary conditions (FP64 ghost fill)
  ChqBC bc;           // homogeneous rules of the correction equation
  ChqTail tail;       // the tail's level table (global pointers filled per block)
  PensLevel lv[kPensMaxLevels];
};
static_assert(sizeof(PensMember) % 8 == 0, "member record is copied as 8-byte words");

struct PensArgs {
  const PensMember *mem;
  const int *order;     // members, largest first
  int count;
  int *queue;           // next position in order
  float *scratch;       // per-block FP32 hierarchies
  long long scratch_stride;
  const double *tol;
  int nu1, nu2, cycles, ramp, max_outer;
  int *state;           // 0 converged, 1 not
  int *corrections;
  int *vcycles;
  double *l2;
  int *nconv;
};

__device__ __forceinline__ ChqG level_g(const PensLevel &L, float *H) {
  ChqG g;
  const long long n = (long long)L.nx * L.ny * L.rz;
  g.u0 = H + L.off;
  g.u1 = g.u0 + n;
  g.b0 = g.u0 + 2 * n;
  g.b1 = g.u0 + 3 * n;
  g.nx = L.nx; g.ny = L.ny; g.nz = L.nz; g.rz = L.rz;
  g.fq = L.fq; g.fy = L.fy;
  return g;
}

// The phases take their level records by reference (to the caller's stack or to shared memory):
// copied into registers they measured slower (35.7 against 27.2 ms for the ensemble config) --
// the extra live registers spill inside the item loops.
template <int NT>
__device__ __noinline__ void b_relax(const ChqG &g, const ChqK &k, const ChqBC &bc, int iterations) {
  const int n = g.nx * g.ny * (g.rz >> 2);
  for (int it = 0; it < iterations; it++)
    for (int color = 0; color < 2; color++) {
      for (int t = threadIdx.x; t < n; t += NT) chq_relax_item<false>(g, k, bc, color, t);
      __syncthreads();
    }
}

// ZU: the fine u is zero and only b is read (chq_restrict_item)
template <int NT, bool ZU = false>
__device__ __noinline__ void b_restrict(const ChqG &f, const ChqG &c, const ChqK &k, const ChqBC &bc, const FDiv &fcm) {
  const int n = c.nx * c.ny * fcm.d;
  for (int t = threadIdx.x; t < n; t += NT) chq_restrict_item<false, ZU>(f, c, k, bc, fcm, t);
  __syncthreads();
}

// MODE: add into the fine u, assign it, or add the result into the FP64 x (chq_prolong_item)
template <int NT, int MODE = CHQ_P_ADD>
__device__ __noinline__ void b_prolong(const ChqG &c, const ChqG &f, const ChqBC &bc, const FDiv &fcm,
                                       ChqX X = ChqX{nullptr, 0, 0}) {
  const int n = c.nx * c.ny * fcm.d;
  for (int t = threadIdx.x; t < n; t += NT) chq_prolong_item<false, MODE>(c, f, bc, fcm, t, X);
  __syncthreads();
}


// r = b - A x in FP64 (the reference operator with the ghost values of x), written as float into
// the level-0 colour arrays; returns the block's sum of r^2 (every thread gets it).
// The FP64 level-0 record of a member.
struct Fine64 {
  double *x;
  const double *b;
  long long xs, ys;
  int nx, ny, nz, M, vec;
  FDiv fM, fY;
};

__device__ __forceinline__ Fine64 fine64(const PensMember &D) {
  Fine64 F;
  F.x = D.x; F.b = D.b; F.xs = D.xs; F.ys = D.ys;
  F.nx = D.nx; F.ny = D.ny; F.nz = D.nz; F.M = D.M; F.vec = D.vec;
  F.fM = D.fM; F.fY = D.fY;
  return F;
}

template <int NT>
__device__ __noinline__ double b_residual(const Fine64 &F, const PensOuter &c, const ChqG &g0, double *red) {
  const int n = F.nx * F.ny * F.M;
  const double *__restrict__ x = F.x;
  const double *__restrict__ b = F.b;
  double acc = 0;
  for (int t = threadIdx.x; t < n; t += NT) {
    int i, j, m, row;
    split(F.fM, t, row, m);
    split(F.fY, row, i, j);
    const long long id = (long long)i * F.xs + (long long)j * F.ys + 2 * m;
    const long long cid = (long long)row * g0.rz + m;
    const bool s = (i + j) & 1;
    float *Bs = s ? g0.b1 : g0.b0;
    float *Bo = s ? g0.b0 : g0.b1;
    if (F.vec) {
      const double2 X = *reinterpret_cast<const double2 *>(x + id), B = *reinterpret_cast<const double2 *>(b + id);
      const double2 YM = *reinterpret_cast<const double2 *>(x + id - F.ys);
      const double2 YP = *reinterpret_cast<const double2 *>(x + id + F.ys);
      const double2 XM = *reinterpret_cast<const double2 *>(x + id - F.xs);
      const double2 XP = *reinterpret_cast<const double2 *>(x + id + F.xs);
      const double zl = x[id - 1], zr = x[id + 2];
      const double r0 = B.x - (c.fzh * (zl + X.y) + c.fyh * (YM.x + YP.x) + c.fxh * (XM.x + XP.x) - c.dg * X.x);
      const double r1 = B.y - (c.fzh * (X.x + zr) + c.fyh * (YM.y + YP.y) + c.fxh * (XM.y + XP.y) - c.dg * X.y);
      Bs[cid] = (float)r0;
      Bo[cid] = (float)r1;
      acc += r0 * r0 + r1 * r1;
    } else {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int k = 2 * m + h;
        if (k < F.nz) {
          const long long q = id + h;
          const double r = b[q] - (c.fzh * (x[q - 1] + x[q + 1]) + c.fyh * (x[q - F.ys] + x[q + F.ys]) +
                                   c.fxh * (x[q - F.xs] + x[q + F.xs]) - c.dg * x[q]);
          (h ? Bo : Bs)[cid] = (float)r;
          acc += r * r;
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < NT / 32; w++) s += red[w];
    red[NT / 32] = s;
  }
  __syncthreads();
  return red[NT / 32];
}

// x += (double) e on the interior (e: the level-0 colour arrays of u)
template <int NT>
__device__ __noinline__ void b_add_correction(const Fine64 &F, const ChqG &g0) {
  const int n = F.nx * F.ny * F.M;
  double *__restrict__ x = F.x;
  for (int t = threadIdx.x; t < n; t += NT) {
    int i, j, m, row;
    split(F.fM, t, row, m);
    split(F.fY, row, i, j);
    const long long id = (long long)i * F.xs + (long long)j * F.ys + 2 * m;
    const long long cid = (long long)row * g0.rz + m;
    const bool s = (i + j) & 1;
    const float e0 = (s ? g0.u1 : g0.u0)[cid], e1 = (s ? g0.u0 : g0.u1)[cid];
    if (F.vec) {
      double2 X = *reinterpret_cast<double2 *>(x + id);
      X.x = X.x + (double)e0;
      X.y = X.y + (double)e1;
      *reinterpret_cast<double2 *>(x + id) = X;
    } else {
      x[id] = x[id] + (double)e0;
      if (2 * m + 1 < F.nz) x[id + 1] = x[id + 1] + (double)e1;
    }
  }
  __syncthreads();
}

template <int NT>
__device__ __noinline__ void b_tail(PensMember &D, float *sm, int fmg) {
  if (threadIdx.x == 0) D.tail.fmg = fmg;
  __syncthreads();
  chq_tail_run(D.tail, D.tail.lv, sm);
  __syncthreads();
}

// One FP32 correction solve of A e = r (r already in level 0's b) and x += e: from a zero
// correction, r restricted to the tail (b alone is read), the tail solved, nested iteration up
// (an assigning prolongation + ramp iterations per level), then `cycles` V-cycles at level 0
// (none: the nested iteration alone), the last prolongation adding into x -- the schedule of
// ChequerMG::enqueue_fmg, block-wide.
template <int NT>
__device__ void b_correction(PensMember &D, float *H, float *sm, const PensArgs &A) {
  const int ts = D.ts;
  if (ts == 0) {  // the whole hierarchy in the tail
    b_tail<NT>(D, sm, 1);
    for (int c = 1; c < A.cycles; c++) b_tail<NT>(D, sm, 0);
    b_add_correction<NT>(fine64(D), level_g(D.lv[0], H));
    return;
  }
  for (int l = 0; l < ts; l++)
    b_restrict<NT, true>(level_g(D.lv[l], H), level_g(D.lv[l + 1], H), D.lv[l].k, D.bc, D.lv[l + 1].fcm);
  b_tail<NT>(D, sm, 1);
  for (int f = ts - 1; f >= 1; f--) {
    b_prolong<NT, CHQ_P_ASSIGN>(level_g(D.lv[f + 1], H), level_g(D.lv[f], H), D.bc, D.lv[f + 1].fcm);
    b_relax<NT>(level_g(D.lv[f], H), D.lv[f].k, D.bc, A.ramp);
  }
  b_prolong<NT, CHQ_P_ASSIGN>(level_g(D.lv[1], H), level_g(D.lv[0], H), D.bc, D.lv[1].fcm);
  if (A.cycles <= 0) {
    b_add_correction<NT>(fine64(D), level_g(D.lv[0], H));
    return;
  }
  for (int c = 0; c < A.cycles; c++) {
    for (int l = 0; l < ts; l++) {
      b_relax<NT>(level_g(D.lv[l], H), D.lv[l].k, D.bc, A.nu1);
      b_restrict<NT>(level_g(D.lv[l], H), level_g(D.lv[l + 1], H), D.lv[l].k, D.bc, D.lv[l + 1].fcm);
    }
    b_tail<NT>(D, sm, 0);
    for (int l = ts - 1; l >= 1; l--) {
      b_prolong<NT>(level_g(D.lv[l + 1], H), level_g(D.lv[l], H), D.bc, D.lv[l + 1].fcm);
      b_relax<NT>(level_g(D.lv[l], H), D.lv[l].k, D.bc, A.nu2);
    }
    if (c < A.cycles - 1) {
      b_prolong<NT>(level_g(D.lv[1], H), level_g(D.lv[0], H), D.bc, D.lv[1].fcm);
    } else {
      const ChqX X{D.x, D.xs, D.ys};
      if (D.vec) b_prolong<NT, CHQ_P_X64V>(level_g(D.lv[1], H), level_g(D.lv[0], H), D.bc, D.lv[1].fcm, X);
      else b_prolong<NT, CHQ_P_X64>(level_g(D.lv[1], H), level_g(D.lv[0], H), D.bc, D.lv[1].fcm, X);
    }
  }
}

// MINB blocks of NT threads per SM: 1024 threads at up to 64 registers, or (dense) 1536 threads
// at up to 42 registers (the transfer phases then spill a little more)
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_pens_solve(const __grid_constant__ PensArgs A) {
  extern __shared__ float sm[];
  __shared__ PensMember D;
  __shared__ double red[NT / 32 + 1];
  __shared__ int s_q;
  float *H = A.scratch + (long long)blockIdx.x * A.scratch_stride;
  for (;;) {
    if (threadIdx.x == 0) s_q = atomicAdd(A.queue, 1);
    __syncthreads();
    const int q = s_q;
    if (q >= A.count) return;  // uniform across the block
    const int m = A.order[q];
    {
      const long long *src = reinterpret_cast<const long long *>(A.mem + m);
      long long *dst = reinterpret_cast<long long *>(&D);
      for (int w = threadIdx.x; w < (int)(sizeof(PensMember) / 8); w += NT) dst[w] = src[w];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int l = 0; l < D.tail.nlev; l++) {
        const ChqG g = level_g(D.lv[D.ts + l], H);
        D.tail.lv[l].gu0 = g.u0;
        D.tail.lv[l].gu1 = g.u1;
        D.tail.lv[l].gb0 = g.b0;
        D.tail.lv[l].gb1 = g.b1;
      }
      D.tail.nu1 = A.nu1;
      D.tail.nu2 = A.nu2;
    }
    __syncthreads();
    const ChqG g0 = level_g(D.lv[0], H);
    const double tol = A.tol[m];
    int corr = 0, conv = 0;
    double l2 = 0;
    for (;;) {
      level1_fill_block<double>(D.x, D.xs, D.ys, D.nx, D.ny, D.nz, D.bcd, D.hx, D.hy, D.hz);
      __syncthreads();
      l2 = sqrt(b_residual<NT>(fine64(D), D.oc, g0, red) * D.inv_n);
      if (l2 <= tol) { conv = 1; break; }
      if (corr >= A.max_outer || !(l2 == l2)) break;
      b_correction<NT>(D, H, sm, A);  // x += e included
      corr++;
    }
    if (threadIdx.x == 0) {
      A.state[m] = conv ? 0 : 1;
      A.corrections[m] = corr;
      A.vcycles[m] = corr * A.cycles;
      A.l2[m] = l2;
      if (conv) atomicAdd(A.nconv, 1);
    }
    __syncthreads();
  }
}

__global__ void k_pens_reset(int *queue, int *nconv) {
  *queue = 0;
  *nconv = 0;
}

template <int NT, int MINB>
void *pens_kernel() {
  return reinterpret_cast<void *>(&k_pens_solve<NT, MINB>);
}

}  // namespace

struct PersistentEnsemble {
  int count = 0;
  ocu_pens_params prm{};
  std::vector<PensMember> host;
  std::vector<ocu_grid> rhs_view, p_view;
  std::vector<long long> cells;
  PensMember *d_mem = nullptr;
  int *d_order = nullptr, *d_ints = nullptr;  // queue, nconv, then state / corrections / vcycles
  double *d_tol = nullptr, *d_l2 = nullptr, *h_tol = nullptr;
  int *h_nconv = nullptr;
  void *fp64 = nullptr;
  float *scratch = nullptr;
  long long scratch_stride = 0;
  size_t scratch_blocks = 0;
  size_t tail_smem = 0;
  int blocks = 0;
  cudaStream_t user = nullptr;
  cudaGraphExec_t graph = nullptr;

  ~PersistentEnsemble() {
    if (user) cudaStreamSynchronize(user);
    else cudaDeviceSynchronize();
    if (graph) cudaGraphExecDestroy(graph);
    cudaFree(d_mem);
    cudaFree(d_order);
    cudaFree(d_ints);
    cudaFree(d_tol);
    cudaFree(d_l2);
    cudaFree(fp64);
    cudaFree(scratch);
    if (h_tol) cudaFreeHost(h_tol);
    if (h_nconv) cudaFreeHost(h_nconv);
  }

  int *d_queue() const { return d_ints; }
  int *d_nconv() const { return d_ints + 1; }
  int *d_state() const { return d_ints + 2; }
  int *d_corr() const { return d_ints + 2 + count; }
  int *d_vc() const { return d_ints + 2 + 2 * count; }

  ocu_status describe(int m, int nx, int ny, int nz, double hx, double hy, double hz, double *x, double *b,
                      const ocu_layout &L, long long *floats) {
    MGCore<double> geo;
    OCU_TRY(geo.set_geometry(prm.bc, false, nx, ny, nz, hx, hy, hz, L));
    ocu_bc_set hb = prm.bc;
    bc_make_homogeneous(&hb);
    if (!ChequerMG::suits(geo.dim, hb))
      return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ocu_pens_create - member %d (%d,%d,%d): the split FP32 hierarchy needs "
                                       "at least two levels and even sizes along periodic axes", m, nx, ny, nz);
    const int L_ = geo.num_levels;
    if (L_ > kPensMaxLevels)
      return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ocu_pens_create - member %d has %d levels (at most %d)", m, L_,
                  kPensMaxLevels);
    PensMember D;
    std::memset(&D, 0, sizeof(D));
    D.x = x;
    D.b = b;
    D.xs = L.xstride;
    D.ys = L.ystride;
    D.nx = nx; D.ny = ny; D.nz = nz;
    D.M = (nz + 1) / 2;
    D.fM = make_fdiv(D.M);
    D.fY = make_fdiv(ny);
    D.nlev = L_;
    D.vec = (nz % 2 == 0 && L.shift % 2 == 0 && L.xstride % 2 == 0 && L.ystride % 2 == 0) ? 1 : 0;
    D.inv_n = 1.0 / ((double)nx * ny * nz);
    D.hx = hx; D.hy = hy; D.hz = hz;
    const double h0 = geo.h[0];
    D.oc.fxh = geo.fx / (h0 * h0);
    D.oc.fyh = geo.fy / (h0 * h0);
    D.oc.fzh = geo.fz / (h0 * h0);
    D.oc.dg = 2 * (geo.fx + geo.fy + geo.fz) / (h0 * h0);
    D.bcd = to_dev(prm.bc);
    D.bc = make_bc(hb, geo.fx, geo.fy, geo.fz);
    long long off = 0;
    for (int l = 0; l < L_; l++) {
      PensLevel &P = D.lv[l];
      P.nx = geo.dim[l][0]; P.ny = geo.dim[l][1]; P.nz = geo.dim[l][2];
      P.rz = round4((P.nz + 1) / 2);
      P.ysh = log2_exact(P.ny);
      P.zsh = log2_exact(P.nz);
      P.fq = make_fdiv(P.rz / 4);
      P.fy = make_fdiv(P.ny);
      P.fcm = make_fdiv((P.nz + 1) / 2);
      P.off = off;
      P.k = make_k(geo.h[l], geo.fx, geo.fy, geo.fz, geo.omega);
      off += 4LL * P.nx * P.ny * P.rz;
    }
    *floats = off;
    // the tail: the coarse levels of ChequerMG's rule
    const int ts = tail_first(geo.dim, prm.tail_cells > 0 ? prm.tail_cells : kChqTailCells);
    D.ts = ts;
    ChqTail &T = D.tail;
    T.nlev = L_ - ts;
    T.level0 = ts == 0;
    T.bc = D.bc;
    {
      const auto &d = geo.dim[L_ - 1];
      const int a = d[0] * d[1], bb = d[1] * d[2], c = d[0] * d[2];
      T.citers = std::max(a, std::max(bb, c)) / 2;
    }
    int soff = 0, largest = 0;
    for (int l = ts; l < L_; l++) {
      const PensLevel &P = D.lv[l];
      SLv &s = T.lv[l - ts];
      s.nx = P.nx; s.ny = P.ny; s.nz = P.nz; s.rz = P.rz;
      s.off = soff;
      s.mlog = log2_exact((P.nz + 1) / 2);
      s.ylog = P.ysh;
      s.nzlog = P.zsh;
      s.k = P.k;
      soff += 4 * P.nx * P.ny * P.rz;
      if (l < L_ - 1 && 2 * P.nx * P.ny * P.rz > largest) largest = 2 * P.nx * P.ny * P.rz;
    }
    T.scratch = soff;
    tail_smem = std::max(tail_smem, (size_t)(soff + largest) * sizeof(float));
    host[m] = D;
    return OCU_OK;
  }

  ocu_status create(int n, const int *dims, const double *h, const ocu_pens_params &p) {
    count = n;
    prm = p;
    if (prm.nu1 < 1 || prm.nu2 < 0 || prm.cycles < 0 || prm.max_outer < 0)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_create - bad smoothing or cycle counts");
    host.resize(n);
    rhs_view.resize(n);
    p_view.resize(n);
    cells.resize(n);
    std::vector<ocu_layout> lay(n);
    std::vector<long long> at(n);
    long long total = 0;
    for (int m = 0; m < n; m++) {
      layout_compute(dims[3 * m], dims[3 * m + 1], dims[3 * m + 2], 1, 1, 1, 0, 0, 0, &lay[m]);
      at[m] = total;
      total += (lay[m].allocated + 31) / 32 * 32;  // 256-byte aligned grids
      cells[m] = (long long)dims[3 * m] * dims[3 * m + 1] * dims[3 * m + 2];
    }
    OCU_TRY(check_cuda(cudaMalloc(&fp64, 2 * sizeof(double) * total), "cudaMalloc (ensemble FP64 grids)"));
    OCU_TRY(check_cuda(cudaMemset(fp64, 0, 2 * sizeof(double) * total), "cudaMemset"));
    double *xb = (double *)fp64, *bb = xb + total;
    long long max_floats = 0;
    for (int m = 0; m < n; m++) {
      double *x = xb + at[m], *b = bb + at[m];
      rhs_view[m] = ocu_grid{OCU_F64, lay[m], b, false};
      p_view[m] = ocu_grid{OCU_F64, lay[m], x, false};
      long long fl = 0;
      OCU_TRY(describe(m, dims[3 * m], dims[3 * m + 1], dims[3 * m + 2], h[3 * m], h[3 * m + 1], h[3 * m + 2],
                       x + lay[m].shift, b + lay[m].shift, lay[m], &fl));
      max_floats = std::max(max_floats, fl);
    }
    scratch_stride = (max_floats + 63) / 64 * 64;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells[a] > cells[b]; });
    OCU_TRY(check_cuda(cudaMalloc(&d_mem, sizeof(PensMember) * n), "cudaMalloc (member records)"));
    OCU_TRY(check_cuda(cudaMemcpy(d_mem, host.data(), sizeof(PensMember) * n, cudaMemcpyHostToDevice), "records"));
    OCU_TRY(check_cuda(cudaMalloc(&d_order, sizeof(int) * n), "cudaMalloc (order)"));
    OCU_TRY(check_cuda(cudaMemcpy(d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "order"));
    OCU_TRY(check_cuda(cudaMalloc(&d_ints, sizeof(int) * (2 + 3 * (size_t)n)), "cudaMalloc (member state)"));
    OCU_TRY(check_cuda(cudaMemset(d_ints, 0, sizeof(int) * (2 + 3 * (size_t)n)), "cudaMemset"));
    OCU_TRY(check_cuda(cudaMalloc(&d_tol, sizeof(double) * n), "cudaMalloc (tolerances)"));
    OCU_TRY(check_cuda(cudaMalloc(&d_l2, sizeof(double) * n), "cudaMalloc (norms)"));
    OCU_TRY(check_cuda(cudaMemset(d_l2, 0, sizeof(double) * n), "cudaMemset"));
    OCU_TRY(check_cuda(cudaMallocHost(&h_tol, sizeof(double) * n), "cudaMallocHost (tolerances)"));
    OCU_TRY(check_cuda(cudaMallocHost(&h_nconv, sizeof(int)), "cudaMallocHost"));
    OCU_TRY(configure());
    return check_cuda(cudaDeviceSynchronize(), "ocu_pens_create");
  }

  void *kernel() const {
    if (prm.dense) return prm.threads == 256 ? pens_kernel<256, 6>() : pens_kernel<512, 3>();
    switch (prm.threads) {
      case 256: return pens_kernel<256, 4>();
      case 1024: return pens_kernel<1024, 1>();
      default: return pens_kernel<512, 2>();
    }
  }

  // Blocks resident at once for the current thread count; the scratch holds one hierarchy each.
  ocu_status configure() {
    if (prm.threads != 256 && prm.threads != 512 && prm.threads != 1024)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens - threads must be 256, 512 or 1024 (got %d)", prm.threads);
    if (prm.dense && prm.threads == 1024)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens - the dense build takes 256 or 512 threads");
    void *k = kernel();
    OCU_TRY(check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tail_smem),
                       "cudaFuncSetAttribute (persistent ensemble)"));
    int dev = 0, sms = 0, per_sm = 0;
    OCU_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
    OCU_TRY(check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count"));
    OCU_TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, prm.threads, tail_smem),
                       "occupancy"));
    if (per_sm < 1) return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ocu_pens - the kernel does not fit on an SM");
    blocks = std::min(per_sm * sms, count);
    if ((size_t)blocks > scratch_blocks) {
      cudaFree(scratch);
      scratch = nullptr;
      OCU_TRY(check_cuda(cudaMalloc(&scratch, sizeof(float) * (size_t)scratch_stride * blocks),
                         "cudaMalloc (FP32 scratch hierarchies)"));
      OCU_TRY(check_cuda(cudaMemset(scratch, 0, sizeof(float) * (size_t)scratch_stride * blocks), "cudaMemset"));
      scratch_blocks = blocks;
    }
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    return OCU_OK;
  }

  ocu_status enqueue(cudaStream_t s) {
    OCU_TRY(check_cuda(cudaMemcpyAsync(d_tol, h_tol, sizeof(double) * count, cudaMemcpyHostToDevice, s),
                       "tolerances"));
    k_pens_reset<<<1, 1, 0, s>>>(d_queue(), d_nconv());
    OCU_TRY(check_launch("k_pens_reset"));
    PensArgs A;
    A.mem = d_mem;
    A.order = d_order;
    A.count = count;
    A.queue = d_queue();
    A.scratch = scratch;
    A.scratch_stride = scratch_stride;
    A.tol = d_tol;
    A.nu1 = prm.nu1;
    A.nu2 = prm.nu2;
    A.cycles = prm.cycles;
    A.ramp = prm.ramp_iters > 0 ? prm.ramp_iters : prm.nu1 + prm.nu2;
    A.max_outer = prm.max_outer > 0 ? prm.max_outer : 10;
    A.state = d_state();
    A.corrections = d_corr();
    A.vcycles = d_vc();
    A.l2 = d_l2;
    A.nconv = d_nconv();
    void *args[] = {&A};
    OCU_TRY(check_cuda(cudaLaunchKernel(kernel(), dim3(blocks), dim3(prm.threads), args, tail_smem, s),
                       "k_pens_solve"));
    return check_cuda(cudaMemcpyAsync(h_nconv, d_nconv(), sizeof(int), cudaMemcpyDeviceToHost, s), "converged count");
  }

  ocu_status solve(const double *tol, int *converged) {
    for (int m = 0; m < count; m++) {
      if (!(tol[m] >= 0)) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_solve - bad tolerance for member %d", m);
      h_tol[m] = tol[m];
    }
    cudaStream_t s = user;
    cudaStream_t own = nullptr;
    if (!s) {  // the legacy stream cannot be captured: a private stream ordered after it
      OCU_TRY(check_cuda(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking), "cudaStreamCreate"));
      OCU_TRY(check_cuda(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize"));
      s = own;
    }
    ocu_status st = OCU_OK;
    if (!graph) {
      if (graph) cudaGraphExecDestroy(graph);
      graph = nullptr;
      cudaGraph_t g = nullptr;
      st = check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
      if (st == OCU_OK) {
        set_capturing(true);
        const ocu_status se = enqueue(s);
        set_capturing(false);
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        st = se != OCU_OK ? se : check_cuda(e, "cudaStreamEndCapture");
        if (st == OCU_OK) st = check_cuda(cudaGraphInstantiate(&graph, g, 0), "cudaGraphInstantiate");
        if (g) cudaGraphDestroy(g);
      }
    }
    if (st == OCU_OK) st = check_cuda(cudaGraphLaunch(graph, s), "cudaGraphLaunch");
    if (st == OCU_OK) {
      count_launch(2);
      st = check_cuda(cudaStreamSynchronize(s), "ocu_pens_solve");
    }
    if (own) cudaStreamDestroy(own);
    if (st != OCU_OK) return st;
    if (converged) *converged = *h_nconv;
    return *h_nconv == count ? OCU_OK : OCU_ERR_NOT_CONVERGED;
  }

  ocu_status stats(int m, ocu_pens_stats *out) const {
    int st = 0, corr = 0, vc = 0;
    double l2 = 0;
    OCU_TRY(check_cuda(cudaMemcpy(&st, d_state() + m, sizeof(int), cudaMemcpyDeviceToHost), "member state"));
    OCU_TRY(check_cuda(cudaMemcpy(&corr, d_corr() + m, sizeof(int), cudaMemcpyDeviceToHost), "member state"));
    OCU_TRY(check_cuda(cudaMemcpy(&vc, d_vc() + m, sizeof(int), cudaMemcpyDeviceToHost), "member state"));
    OCU_TRY(check_cuda(cudaMemcpy(&l2, d_l2 + m, sizeof(double), cudaMemcpyDeviceToHost), "member state"));
    out->converged = st == 0;
    out->corrections = corr;
    out->vcycles = vc;
    out->l2 = l2;
    return OCU_OK;
  }

  ocu_status clear_pressures(cudaStream_t s) {
    for (int m = 0; m < count; m++)
      OCU_TRY(check_cuda(cudaMemsetAsync(p_view[m].buf, 0, sizeof(double) * p_view[m].L.allocated, s), "cudaMemset"));
    return OCU_OK;
  }

  // Times whole solves from a zero guess over thread counts, correction schedules and smoothing
  // pairs; keeps the fastest that converges every member; leaves every pressure zeroed.
  ocu_status autotune(const double *tol) {
    const ocu_pens_params base = prm;
    struct Cand { int threads, dense, cycles, nu1, nu2; };
    std::vector<Cand> cands;
    for (auto sh : {std::make_pair(256, 0), std::make_pair(512, 0), std::make_pair(1024, 0), std::make_pair(256, 1),
                    std::make_pair(512, 1)})
      for (int cy : {0, 1, 2, 3})
        for (auto nu : {std::make_pair(2, 2), std::make_pair(2, 1), std::make_pair(1, 1)})
          cands.push_back({sh.first, sh.second, cy, nu.first, nu.second});
    cudaStream_t s = user;
    double best = 1e300;
    ocu_pens_params best_p = base;
    cudaEvent_t e0, e1;
    OCU_TRY(check_cuda(cudaEventCreate(&e0), "cudaEventCreate"));
    OCU_TRY(check_cuda(cudaEventCreate(&e1), "cudaEventCreate"));
    ocu_status st = OCU_OK;
    for (const Cand &c : cands) {
      prm = base;
      prm.threads = c.threads;
      prm.dense = c.dense;
      prm.cycles = c.cycles;
      prm.nu1 = c.nu1;
      prm.nu2 = c.nu2;
      if ((st = configure()) != OCU_OK) break;
      double ms = 1e300;
      bool all = true;
      for (int rep = 0; rep < 2 && all; rep++) {
        if ((st = clear_pressures(s)) != OCU_OK) break;
        int conv = 0;
        cudaEventRecord(e0, s);
        const ocu_status ss = solve(tol, &conv);
        cudaEventRecord(e1, s);
        if (ss != OCU_OK && ss != OCU_ERR_NOT_CONVERGED) { st = ss; break; }
        cudaEventSynchronize(e1);
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        ms = std::min(ms, (double)t);
        all = conv == count;
      }
      if (st != OCU_OK) break;
      if (all && ms < best) {
        best = ms;
        best_p = prm;
        best_p.ms = ms;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != OCU_OK) return st;
    prm = best_p;
    OCU_TRY(configure());
    OCU_TRY(clear_pressures(s));
    return check_cuda(cudaStreamSynchronize(s), "ocu_pens_autotune");
  }

  ocu_status set_params(const ocu_pens_params &p) {
    if (p.nu1 < 1 || p.nu2 < 0 || p.cycles < 0 || p.max_outer < 0)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_set_params - bad smoothing or cycle counts");
    if (p.tail_cells != prm.tail_cells)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_set_params - tail_cells is fixed at creation");
    const ocu_bc_set bc = prm.bc;
    const int old_threads = prm.threads, old_dense = prm.dense;
    prm = p;
    prm.bc = bc;  // fixed at creation
    if (graph) {  // counts are launch arguments baked into the graph
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    if (prm.threads != old_threads || prm.dense != old_dense) return configure();
    return OCU_OK;
  }
};

}  // namespace ocub

// ---- C ABI ----------------------------------------------------------------------------------
struct ocu_pens {
  std::unique_ptr<ocub::PersistentEnsemble> impl;
};

using namespace ocub;

#define PENS_CHECK(e)                                                                                  \
  do {                                                                                                 \
    if (!(e) || !(e)->impl) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] persistent ensemble - null handle"); \
  } while (0)

extern "C" {

void ocu_pens_params_default(ocu_pens_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  ocu_bc nb{OCU_BC_NEUMANN, 0.0, 0.0};
  p->bc.xpos = p->bc.xneg = p->bc.ypos = p->bc.yneg = p->bc.zpos = p->bc.zneg = nb;
  p->nu1 = 2;
  p->nu2 = 2;
  p->cycles = 2;
  p->ramp_iters = 0;
  p->max_outer = 10;
  p->threads = 512;
  p->dense = 0;
  p->tail_cells = 0;
  p->ms = 0;
}

ocu_status ocu_pens_create(int members, const int *dims, const double *h, const ocu_pens_params *params,
                           ocu_pens **out) {
  if (!out || !dims || !h) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_create - null argument");
  *out = nullptr;
  if (members < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_create - members must be >= 1");
  for (int m = 0; m < members; m++) {
    if (dims[3 * m] < 2 || dims[3 * m + 1] < 2 || dims[3 * m + 2] < 2)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_create - member %d has bad dimensions", m);
    for (int a = 0; a < 3; a++)
      if (!(h[3 * m + a] > 0) || !std::isfinite(h[3 * m + a]))
        return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_create - member %d has a bad spacing", m);
  }
  ocu_pens_params p;
  if (params) p = *params; else ocu_pens_params_default(&p);
  std::unique_ptr<ocu_pens> e(new ocu_pens());
  e->impl.reset(new PersistentEnsemble());
  OCU_TRY(e->impl->create(members, dims, h, p));
  *out = e.release();
  return OCU_OK;
}

void ocu_pens_destroy(ocu_pens *e) { delete e; }

ocu_status ocu_pens_set_stream(ocu_pens *e, ocu_stream s) {
  PENS_CHECK(e);
  if (e->impl->user != (cudaStream_t)s && e->impl->graph) {
    cudaGraphExecDestroy(e->impl->graph);
    e->impl->graph = nullptr;
  }
  e->impl->user = (cudaStream_t)s;
  return OCU_OK;
}

ocu_status ocu_pens_rhs(ocu_pens *e, int member, ocu_grid **out) {
  PENS_CHECK(e);
  if (!out || member < 0 || member >= e->impl->count)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_rhs - bad member");
  *out = &e->impl->rhs_view[member];
  return OCU_OK;
}

ocu_status ocu_pens_pressure(ocu_pens *e, int member, ocu_grid **out) {
  PENS_CHECK(e);
  if (!out || member < 0 || member >= e->impl->count)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_pressure - bad member");
  *out = &e->impl->p_view[member];
  return OCU_OK;
}

ocu_status ocu_pens_solve(ocu_pens *e, const double *tol, int *converged) {
  PENS_CHECK(e);
  if (!tol) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_solve - null tolerances");
  return e->impl->solve(tol, converged);
}

ocu_status ocu_pens_member_stats(const ocu_pens *e, int member, ocu_pens_stats *stats) {
  PENS_CHECK(e);
  if (!stats || member < 0 || member >= e->impl->count)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_member_stats - bad member");
  return e->impl->stats(member, stats);
}

ocu_status ocu_pens_get_params(const ocu_pens *e, ocu_pens_params *p) {
  PENS_CHECK(e);
  if (!p) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_get_params - null argument");
  *p = e->impl->prm;
  return OCU_OK;
}

ocu_status ocu_pens_set_params(ocu_pens *e, const ocu_pens_params *p) {
  PENS_CHECK(e);
  if (!p) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_set_params - null argument");
  return e->impl->set_params(*p);
}

ocu_status ocu_pens_launch_shape(const ocu_pens *e, int *blocks, int *threads, long long *scratch_bytes) {
  PENS_CHECK(e);
  if (blocks) *blocks = e->impl->blocks;
  if (threads) *threads = e->impl->prm.threads;
  if (scratch_bytes) *scratch_bytes = (long long)sizeof(float) * e->impl->scratch_stride * e->impl->scratch_blocks;
  return OCU_OK;
}

ocu_status ocu_pens_autotune(ocu_pens *e, const double *tol) {
  PENS_CHECK(e);
  if (!tol) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pens_autotune - null tolerances");
  return e->impl->autotune(tol);
}

}  // extern "C"
