// Sol_PCGPressure3DDevice<T> (ocuequation/sol_pcgpressure3d.h:41-97, sol_pcgpressure3d.cu):
// conjugate gradients on L p = rhs, L = -div(c grad) with a cell coefficient grid c, and the
// reference's four preconditioners.  The kernels keep the reference's expressions and operand
// order (the f/h^2 factors are T values passed as double, so each product is evaluated in double
// on T operands and rounded to T once); the dot products fold the pointwise products in the
// reference's reduce_sum order without storing the product grid; the multigrid preconditioner
// is this library's multigrid solver (run_fmg / run_vcycles, bit-identical to the reference's).
// The CG scalars are T on the host, read back per dot product as the reference does.
#include <cmath>
#include <cstring>
#include <memory>

#include "mg_solver.h"
#include "ocu_internal.h"

namespace ocub {

namespace {

constexpr int kPcgCellsI = 4;  // cells along i per thread (their loads in flight together)

// apply_laplacian (sol_pcgpressure3d.cu:83-117)
template <typename T>
__global__ void __launch_bounds__(256) k_pcg_laplacian(T *__restrict__ dst, const T *__restrict__ src,
                                                       const T *__restrict__ coef, double fxh, double fyh, double fzh,
                                                       long long xs, long long ys, int nx, int ny, int nz) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (k >= nz || j >= ny) return;
#pragma unroll
  for (int ci = 0; ci < kPcgCellsI; ci++) {
    const int i = blockIdx.z * kPcgCellsI + ci;
    if (i >= nx) break;
    const long long id = (long long)i * xs + (long long)j * ys + k;
    const T c = src[id], cc = coef[id];
    dst[id] = (T)(-(fzh * (src[id - 1] - c) * (T)0.5 * (coef[id - 1] + cc) +
                    fzh * (src[id + 1] - c) * (T)0.5 * (coef[id + 1] + cc) +
                    fyh * (src[id - ys] - c) * (T)0.5 * (coef[id - ys] + cc) +
                    fyh * (src[id + ys] - c) * (T)0.5 * (coef[id + ys] + cc) +
                    fxh * (src[id - xs] - c) * (T)0.5 * (coef[id - xs] + cc) +
                    fxh * (src[id + xs] - c) * (T)0.5 * (coef[id + xs] + cc)));
  }
}

// diag_preconditioner (sol_pcgpressure3d.cu:43-79); dst may be src
template <typename T>
__global__ void __launch_bounds__(256) k_pcg_diag(T *dst, const T *src, const T *__restrict__ coef, double fxh,
                                                  double fyh, double fzh, long long xs, long long ys, int nx, int ny,
                                                  int nz) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (k >= nz || j >= ny) return;
#pragma unroll
  for (int ci = 0; ci < kPcgCellsI; ci++) {
    const int i = blockIdx.z * kPcgCellsI + ci;
    if (i >= nx) break;
    const long long id = (long long)i * xs + (long long)j * ys + k;
    const T cc = coef[id];
    const T diagonal = (T)(fzh * (T)0.5 * (coef[id - 1] + cc) + fzh * (T)0.5 * (coef[id + 1] + cc) +
                           fyh * (T)0.5 * (coef[id - ys] + cc) + fyh * (T)0.5 * (coef[id + ys] + cc) +
                           fxh * (T)0.5 * (coef[id - xs] + cc) + fxh * (T)0.5 * (coef[id + xs] + cc));
    dst[id] = src[id] / diagonal;
  }
}

inline void pcg_shape(int nx, int ny, int nz, dim3 *grid, dim3 *block) {
  *block = nz >= 64 ? dim3(64, 4) : dim3(32, 8);
  *grid = dim3((nz + block->x - 1) / block->x, (ny + block->y - 1) / block->y, (nx + kPcgCellsI - 1) / kPcgCellsI);
}

}  // namespace

struct PCGSolver {
  ocu_dtype dtype;
  ocu_pcg_params prm;
  int nx = 0, ny = 0, nz = 0;
  double h = 1, fx = 0, fy = 0, fz = 0;
  ocu_grid *rhs = nullptr, *coef = nullptr;   // borrowed
  ocu_grid *p = nullptr, *r = nullptr, *y = nullptr, *d = nullptr;
  std::unique_ptr<ocu_mg> mg;
  void *scratch = nullptr;
  double *d_red = nullptr, *h_red = nullptr;
  cudaStream_t stream = nullptr;
  int iterations = 0;
  bool initialized = false;

  explicit PCGSolver(ocu_dtype dt, const ocu_pcg_params &p_) : dtype(dt), prm(p_) {}
  ~PCGSolver() {
    if (stream) cudaStreamSynchronize(stream);
    for (ocu_grid *g : {p, r, y, d})
      if (g) {
        cudaFree(g->buf);
        delete g;
      }
    cudaFree(scratch);
    cudaFree(d_red);
    if (h_red) cudaFreeHost(h_red);
  }

  size_t es() const { return dtype == OCU_F64 ? 8 : 4; }
  double hx() const { return h / std::sqrt(fx); }
  double hy() const { return h / std::sqrt(fy); }
  double hz() const { return h / std::sqrt(fz); }
  // the reference's host code holds f/h^2 in T
  double fh(double f) const { return dtype == OCU_F64 ? f / (h * h) : (double)(float)(f / (h * h)); }
  double round_t(double x) const { return dtype == OCU_F64 ? x : (double)(float)x; }

  ocu_status alloc(ocu_grid **g) {
    *g = new ocu_grid{dtype, rhs->L, nullptr, true};
    OCU_TRY(check_cuda(cudaMalloc(&(*g)->buf, es() * rhs->L.allocated), "cudaMalloc(pcg)"));
    return check_cuda(cudaMemset((*g)->buf, 0, es() * rhs->L.allocated), "cudaMemset(pcg)");
  }

  // initialize_storage (sol_pcgpressure3d.cu:604-654)
  ocu_status initialize_storage(int nx_, int ny_, int nz_, float hxv, float hyv, float hzv, ocu_grid *rhs_,
                                ocu_grid *coef_) {
    if (initialized) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_PCGPressure3DDevice::initialize_storage - already initialized");
    if (!std::isfinite(hxv) || !std::isfinite(hyv) || !std::isfinite(hzv))
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_PCGPressure3DDevice::initialize_storage - garbage hx,hy,hz value %f %f %f", hxv, hyv, hzv);
    const ocu_bc *f[6] = {&prm.bc.xpos, &prm.bc.xneg, &prm.bc.ypos, &prm.bc.yneg, &prm.bc.zpos, &prm.bc.zneg};
    for (int q = 0; q < 6; q++)
      if (f[q]->type != OCU_BC_PERIODIC && f[q]->type != OCU_BC_NEUMANN)
        return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_PCGPressure3DDevice::initialize_storage - unsupported boundary type");
    if (!rhs_ || !coef_ || rhs_->dtype != dtype || coef_->dtype != dtype)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_PCGPressure3DDevice::initialize_storage - rhs / coefficient type");
    if (rhs_->L.gx < 1 || rhs_->L.gy < 1 || rhs_->L.gz < 1)
      return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_MultigridPressure3DDevice::initialize_storage - rhs has invalid ghost cells (%d,%d,%d), must be >= 1", rhs_->L.gx, rhs_->L.gy, rhs_->L.gz);
    if (rhs_->L.nx != nx_ || rhs_->L.ny != ny_ || rhs_->L.nz != nz_)
      return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_MultigridPressure3DDevice::initialize_storage - rhs dimension mismatch");
    if (!layout_match(coef_->L, rhs_->L))
      return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_MultigridPressure3DDevice::initialize_storage - coefficient layout must match rhs");
    h = std::min(std::min((double)hxv, (double)hyv), (double)hzv);
    fx = (h * h) / ((double)hxv * hxv);
    fy = (h * h) / ((double)hyv * hyv);
    fz = (h * h) / ((double)hzv * hzv);
    nx = nx_; ny = ny_; nz = nz_;
    rhs = rhs_;
    coef = coef_;
    for (ocu_grid **g : {&p, &r, &y, &d}) OCU_TRY(alloc(g));
    ocu_mg_params mp;
    ocu_mg_params_default(&mp);
    mp.bc = prm.bc;
    mp.nu1 = 2;
    mp.nu2 = 2;
    mp.convergence = OCU_CONVERGENCE_NONE_CALC_L2LINF;
    mg.reset(new ocu_mg(dtype == OCU_F64 ? OCU_MG_F64 : OCU_MG_F32, mp));
    mg->s.set_stream(stream);
    OCU_TRY(mg->s.initialize_storage(nx, ny, nz, hxv, hyv, hzv, r));
    const size_t sb = reduce_scratch_bytes(rhs->L, es());
    OCU_TRY(check_cuda(cudaMalloc(&scratch, sb), "cudaMalloc(pcg scratch)"));
    OCU_TRY(check_cuda(cudaMemset(scratch, 0, sb), "cudaMemset"));
    OCU_TRY(check_cuda(cudaMalloc(&d_red, 2 * sizeof(double)), "cudaMalloc"));
    OCU_TRY(check_cuda(cudaMallocHost(&h_red, 2 * sizeof(double)), "cudaMallocHost"));
    initialized = true;
    return check_cuda(cudaDeviceSynchronize(), "Sol_PCGPressure3DDevice::initialize_storage");
  }

  template <typename T>
  ocu_status bc(ocu_grid *g) {
    return launch_bc_nocorners_dev<T>(origin<T>(g), g->L, prm.bc, hx(), hy(), hz(), stream);
  }

  template <typename T>
  ocu_status apply_laplacian(ocu_grid *dst, ocu_grid *src) {
    OCU_TRY(bc<T>(src));
    dim3 g, b;
    pcg_shape(nx, ny, nz, &g, &b);
    launch_pdl(k_pcg_laplacian<T>, g, b, 0, stream, origin<T>(dst), (const T *)origin<T>(src),
               (const T *)origin<T>(coef), fh(fx), fh(fy), fh(fz), (long long)src->L.xstride,
               (long long)src->L.ystride, nx, ny, nz);
    return check_launch("k_pcg_laplacian");
  }

  template <typename T>
  ocu_status diag(ocu_grid *dst, ocu_grid *src) {
    dim3 g, b;
    pcg_shape(nx, ny, nz, &g, &b);
    launch_pdl(k_pcg_diag<T>, g, b, 0, stream, origin<T>(dst), (const T *)origin<T>(src), (const T *)origin<T>(coef),
               fh(fx), fh(fy), fh(fz), (long long)src->L.xstride, (long long)src->L.ystride, nx, ny, nz);
    return check_launch("k_pcg_diag");
  }

  // <a, b> in T (read back, as the reference's reduce_sum result)
  template <typename T>
  ocu_status dot(ocu_grid *a, ocu_grid *b, double *out) {
    OCU_TRY(launch_dot<T>(origin<T>(a), origin<T>(b), a->L, scratch, d_red, stream));
    OCU_TRY(launch_readback(d_red, h_red, 1, stream));
    OCU_TRY(check_cuda(cudaStreamSynchronize(stream), "dot"));
    *out = h_red[0];
    return OCU_OK;
  }

  template <typename T>
  ocu_status lincomb2(ocu_grid *res, double a1, ocu_grid *g1, double a2, ocu_grid *g2) {
    return launch_lincomb2<T>((T *)res->buf, res->L, (T)a1, (const T *)g1->buf, (T)a2, (const T *)g2->buf, stream);
  }

  // apply_preconditioner (sol_pcgpressure3d.cu:289-331): the multigrid solves for its own
  // right-hand side, the residual grid r
  template <typename T>
  ocu_status precondition(ocu_grid *dst, ocu_grid *src) {
    const int pc = prm.preconditioner;
    if (pc == OCU_PRECOND_JACOBI) return diag<T>(dst, src);
    if (pc == OCU_PRECOND_MULTIGRID || pc == OCU_PRECOND_BFBT) {
      ocu_grid *u = mg->s.pressure;
      OCU_TRY(check_cuda(cudaMemsetAsync(u->buf, 0, es() * u->L.allocated, stream), "clear_zero"));
      const ocu_status st = prm.multigrid_use_fmg ? mg->s.run_fmg(prm.multigrid_cycles)
                                                  : mg->s.run_vcycles(prm.multigrid_cycles);
      if (st != OCU_OK && st != OCU_ERR_NOT_CONVERGED) return st;
      OCU_TRY(launch_lincomb1<T>((T *)dst->buf, (T)-1, (const T *)u->buf, dst->L.allocated, stream));
      if (pc == OCU_PRECOND_BFBT) return diag<T>(dst, dst);
      return OCU_OK;
    }
    return check_cuda(cudaMemcpyAsync(dst->buf, src->buf, es() * src->L.allocated, cudaMemcpyDeviceToDevice, stream),
                      "copy_all_data");
  }

  // do_pcg (sol_pcgpressure3d.cu:335-457)
  template <typename T>
  ocu_status do_pcg(double tolerance, int max_iter, double *rl2, double *rlinf) {
    OCU_TRY(bc<T>(coef));
    OCU_TRY(apply_laplacian<T>(y, p));
    OCU_TRY(lincomb2<T>(r, 1.0, rhs, -1.0, y));
    OCU_TRY(precondition<T>(d, r));
    double delta0, deltanew, deltaold, d_dot_y;
    OCU_TRY(dot<T>(r, d, &delta0));
    deltanew = delta0;
    int it = 0;
    bool converged = (it > max_iter) || (delta0 < tolerance * tolerance);
    while (!converged) {
      OCU_TRY(apply_laplacian<T>(y, d));
      OCU_TRY(dot<T>(d, y, &d_dot_y));
      const double alpha = round_t(deltanew / d_dot_y);
      OCU_TRY(lincomb2<T>(p, 1.0, p, alpha, d));
      if (it % 25 == 0) {  // every 25 iterations the residual is recomputed
        OCU_TRY(apply_laplacian<T>(y, p));
        OCU_TRY(lincomb2<T>(r, 1.0, rhs, -1.0, y));
      } else {
        OCU_TRY(lincomb2<T>(r, 1.0, r, -alpha, y));
      }
      OCU_TRY(precondition<T>(y, r));
      deltaold = deltanew;
      OCU_TRY(dot<T>(r, y, &deltanew));
      const double beta = round_t(deltanew / deltaold);
      OCU_TRY(lincomb2<T>(d, beta, d, 1.0, y));
      it++;
      converged = (it > max_iter) || (deltanew < tolerance * tolerance);
    }
    iterations = it;
    OCU_TRY(launch_reduce<T>(origin<T>(r), r->L, OCU_REDUCE_MAXABS, scratch, d_red + 1, stream));
    OCU_TRY(launch_readback(d_red + 1, h_red + 1, 1, stream));
    OCU_TRY(check_cuda(cudaStreamSynchronize(stream), "linf"));
    *rl2 = std::sqrt(deltanew);
    *rlinf = h_red[1];
    return deltanew <= tolerance * tolerance ? OCU_OK : OCU_ERR_NOT_CONVERGED;
  }

  // solve (sol_pcgpressure3d.cu:571-601)
  ocu_status solve(double *residual, double tolerance, int max_iter) {
    if (!initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] Sol_PCGPressure3DDevice::solve - not initialized");
    if (!std::isfinite((float)tolerance))
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_PCGPressure3DDevice::solve - garbage tolerance value %f", tolerance);
    if (tolerance < 0)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Sol_PCGPressure3DDevice::solve - negative tolerance value %f", tolerance);
    if (max_iter <= 0)
      return fail(OCU_ERR_INVALID_VALUE, "[WARNING] Sol_PCGPressure3DDevice::solve - non-positive max_iter %d", max_iter);
    double l2 = 0, linf = 0;
    const ocu_status st = dtype == OCU_F64 ? do_pcg<double>(tolerance, max_iter, &l2, &linf)
                                           : do_pcg<float>(tolerance, max_iter, &l2, &linf);
    if (st != OCU_OK && st != OCU_ERR_NOT_CONVERGED) return st;
    if (residual) *residual = prm.convergence == OCU_CONVERGENCE_L2 ? l2 : linf;
    return st;
  }
};

}  // namespace ocub

// ---- C ABI ----------------------------------------------------------------------------------
struct ocu_pcg {
  std::unique_ptr<ocub::PCGSolver> impl;
};

using namespace ocub;

#define PCG_CHECK(x)                                                                            \
  do {                                                                                          \
    if (!(x) || !(x)->impl) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] pcg - null handle");      \
  } while (0)

static bool pcg_params_ok(const ocu_pcg_params &p) {
  return (p.convergence == OCU_CONVERGENCE_L2 || p.convergence == OCU_CONVERGENCE_LINF) && p.preconditioner >= 0 &&
         p.preconditioner <= OCU_PRECOND_BFBT && p.multigrid_cycles >= 0;
}

extern "C" {

void ocu_pcg_params_default(ocu_pcg_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  const ocu_bc nb{OCU_BC_NEUMANN, 0.0f, 0.0f};
  p->bc.xpos = p->bc.xneg = p->bc.ypos = p->bc.yneg = p->bc.zpos = p->bc.zneg = nb;
  p->convergence = OCU_CONVERGENCE_L2;
  p->preconditioner = OCU_PRECOND_BFBT;
  p->multigrid_cycles = 2;
  p->multigrid_use_fmg = 1;
}

ocu_status ocu_pcg_create(ocu_dtype dtype, const ocu_pcg_params *params, ocu_pcg **out) {
  if (!out) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pcg_create - null argument");
  *out = nullptr;
  if (dtype != OCU_F32 && dtype != OCU_F64) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pcg_create - bad dtype");
  ocu_pcg_params p;
  if (params) p = *params; else ocu_pcg_params_default(&p);
  if (!pcg_params_ok(p)) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pcg_create - bad parameters");
  std::unique_ptr<ocu_pcg> s(new ocu_pcg());
  s->impl.reset(new PCGSolver(dtype, p));
  *out = s.release();
  return OCU_OK;
}

void ocu_pcg_destroy(ocu_pcg *s) { delete s; }

ocu_status ocu_pcg_set_stream(ocu_pcg *s, ocu_stream stream) {
  PCG_CHECK(s);
  s->impl->stream = (cudaStream_t)stream;
  if (s->impl->mg) s->impl->mg->s.set_stream((cudaStream_t)stream);
  return OCU_OK;
}

ocu_status ocu_pcg_set_params(ocu_pcg *s, const ocu_pcg_params *params) {
  PCG_CHECK(s);
  if (!params || !pcg_params_ok(*params)) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pcg_set_params - bad parameters");
  const ocu_bc_set bc = s->impl->prm.bc;
  s->impl->prm = *params;
  if (s->impl->initialized) s->impl->prm.bc = bc;  // fixed once the storage exists
  return OCU_OK;
}

ocu_status ocu_pcg_initialize_storage(ocu_pcg *s, int nx, int ny, int nz, float hx, float hy, float hz,
                                      ocu_grid *rhs, ocu_grid *coefficient) {
  PCG_CHECK(s);
  return s->impl->initialize_storage(nx, ny, nz, hx, hy, hz, rhs, coefficient);
}

ocu_status ocu_pcg_solve(ocu_pcg *s, double *residual, double tolerance, int max_iter) {
  PCG_CHECK(s);
  return s->impl->solve(residual, tolerance, max_iter);
}

ocu_status ocu_pcg_pressure(ocu_pcg *s, ocu_grid **out) {
  PCG_CHECK(s);
  if (!out) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pcg_pressure - null argument");
  if (!s->impl->initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] ocu_pcg_pressure - not initialized");
  *out = s->impl->p;
  return OCU_OK;
}

ocu_status ocu_pcg_iterations(const ocu_pcg *s, int *out) {
  PCG_CHECK(s);
  if (!out) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_pcg_iterations - null argument");
  *out = s->impl->iterations;
  return OCU_OK;
}

}  // extern "C"
