// extern "C" entry points of libocu_b200.so (declared in include/ocu_b200.h).
#include <cstring>
#include <new>

#include "flow_solvers.h"

using namespace ocub;


#define OCU_NOT_NULL(p, name) \
  if (!(p)) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] %s - null %s", __func__, name)

extern "C" {

const char *ocu_last_error(void) { return ocub::last_error_text(); }

const char *ocu_version(void) { return "opencurrent-b200 0.1 (sm_100a)"; }

unsigned long long ocu_kernel_launch_count(void) { return ocub::launch_count(); }

ocu_status ocu_layout_compute(int nx, int ny, int nz, int gx, int gy, int gz, int padx, int pady, int padz,
                              ocu_layout *out) {
  OCU_NOT_NULL(out, "layout");
  if (nx < 0 || ny < 0 || nz < 0 || gx < 0 || gy < 0 || gz < 0 || padx < 0 || pady < 0 || padz < 0 || gz > 16)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] Grid3DDevice::init - invalid dimensions");
  layout_compute(nx, ny, nz, gx, gy, gz, padx, pady, padz, out);
  return OCU_OK;
}

ocu_status ocu_grid_create(ocu_dtype dtype, int nx, int ny, int nz, int gx, int gy, int gz, int padx, int pady,
                           int padz, ocu_grid **out) {
  OCU_NOT_NULL(out, "out");
  *out = nullptr;
  if (dtype != OCU_F32 && dtype != OCU_F64) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_grid_create - bad dtype");
  ocu_layout L;
  OCU_TRY(ocu_layout_compute(nx, ny, nz, gx, gy, gz, padx, pady, padz, &L));
  ocu_grid *g = new (std::nothrow) ocu_grid{dtype, L, nullptr, true};
  if (!g) return fail(OCU_ERR_ALLOC, "[ERROR] ocu_grid_create - out of host memory");
  cudaError_t e = cudaMalloc(&g->buf, dtype_size(dtype) * L.allocated);
  if (e != cudaSuccess) {
    delete g;
    check_cuda(e, "[ERROR] Grid3DDevice::init - cudaMalloc failed");
    return e == cudaErrorMemoryAllocation ? OCU_ERR_ALLOC : OCU_ERR_CUDA;
  }
  e = cudaMemset(g->buf, 0, dtype_size(dtype) * L.allocated);
  if (e != cudaSuccess) {
    cudaFree(g->buf);
    delete g;
    return check_cuda(e, "cudaMemset");
  }
  *out = g;
  return OCU_OK;
}

ocu_status ocu_grid_wrap(ocu_dtype dtype, const ocu_layout *layout, void *device_buffer, ocu_grid **out) {
  OCU_NOT_NULL(out, "out");
  OCU_NOT_NULL(layout, "layout");
  OCU_NOT_NULL(device_buffer, "device_buffer");
  *out = new (std::nothrow) ocu_grid{dtype, *layout, device_buffer, false};
  return *out ? OCU_OK : fail(OCU_ERR_ALLOC, "[ERROR] ocu_grid_wrap - out of host memory");
}

void ocu_grid_destroy(ocu_grid *g) {
  if (!g) return;
  if (g->owned && g->buf) cudaFree(g->buf);
  delete g;
}

ocu_status ocu_grid_info(const ocu_grid *g, ocu_layout *layout, ocu_dtype *dtype, void **device_buffer) {
  OCU_NOT_NULL(g, "grid");
  if (layout) *layout = g->L;
  if (dtype) *dtype = g->dtype;
  if (device_buffer) *device_buffer = g->buf;
  return OCU_OK;
}

ocu_status ocu_grid_upload_async(ocu_grid *g, const void *host, ocu_stream s) {
  OCU_NOT_NULL(g, "grid");
  OCU_NOT_NULL(host, "host buffer");
  return check_cuda(cudaMemcpyAsync(g->buf, host, dtype_size(g->dtype) * g->L.allocated, cudaMemcpyHostToDevice,
                                    (cudaStream_t)s),
                    "Grid3DDevice::copy_all_data(HostToDevice)");
}

ocu_status ocu_grid_download_async(const ocu_grid *g, void *host, ocu_stream s) {
  OCU_NOT_NULL(g, "grid");
  OCU_NOT_NULL(host, "host buffer");
  return check_cuda(cudaMemcpyAsync(host, g->buf, dtype_size(g->dtype) * g->L.allocated, cudaMemcpyDeviceToHost,
                                    (cudaStream_t)s),
                    "Grid3DHost::copy_all_data(DeviceToHost)");
}

ocu_status ocu_grid_upload(ocu_grid *g, const void *host, ocu_stream s) {
  OCU_TRY(ocu_grid_upload_async(g, host, s));
  return check_cuda(cudaStreamSynchronize((cudaStream_t)s), "upload");
}

ocu_status ocu_grid_download(const ocu_grid *g, void *host, ocu_stream s) {
  OCU_TRY(ocu_grid_download_async(g, host, s));
  return check_cuda(cudaStreamSynchronize((cudaStream_t)s), "download");
}

ocu_status ocu_grid_copy_all_data(ocu_grid *dst, const ocu_grid *src, ocu_stream s) {
  OCU_NOT_NULL(dst, "dst");
  OCU_NOT_NULL(src, "src");
  if (!layout_match(dst->L, src->L))
    return fail(OCU_ERR_LAYOUT, "[ERROR] Grid3DDevice::copy_all_data - mismatch: (%d, %d, %d) != (%d, %d, %d)", dst->L.pnx,
                dst->L.pny, dst->L.pnz, src->L.pnx, src->L.pny, src->L.pnz);
  cudaStream_t st = (cudaStream_t)s;
  const long long n = dst->L.allocated;
  if (dst->dtype == src->dtype)
    return check_cuda(cudaMemcpyAsync(dst->buf, src->buf, dtype_size(dst->dtype) * n, cudaMemcpyDeviceToDevice, st),
                      "cudaMemcpy(DeviceToDevice)");
  if (dst->dtype == OCU_F32) return launch_convert<float, double>((float *)dst->buf, (const double *)src->buf, n, st);
  return launch_convert<double, float>((double *)dst->buf, (const float *)src->buf, n, st);
}

ocu_status ocu_grid_clear(ocu_grid *g, double value, ocu_stream s) {
  OCU_NOT_NULL(g, "grid");
  if (value == 0.0)
    return check_cuda(cudaMemsetAsync(g->buf, 0, dtype_size(g->dtype) * g->L.allocated, (cudaStream_t)s), "cudaMemset");
  if (g->dtype == OCU_F64) return launch_clear<double>((double *)g->buf, g->L.allocated, value, (cudaStream_t)s);
  return launch_clear<float>((float *)g->buf, g->L.allocated, (float)value, (cudaStream_t)s);
}

ocu_status ocu_grid_linear_combination(ocu_grid *res, double a1, const ocu_grid *g1, double a2, const ocu_grid *g2,
                                       ocu_stream s) {
  OCU_NOT_NULL(res, "result");
  OCU_NOT_NULL(g1, "g1");
  if (!layout_match(res->L, g1->L) || (g2 && !layout_match(res->L, g2->L)))
    return fail(OCU_ERR_LAYOUT, "[ERROR] Grid3DDevice::linear_combination - layout mismatch");
  if (res->dtype != g1->dtype || (g2 && res->dtype != g2->dtype))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] linear_combination - element type mismatch");
  cudaStream_t st = (cudaStream_t)s;
  if (res->dtype == OCU_F64) {
    if (!g2) return launch_lincomb1<double>((double *)res->buf, a1, (const double *)g1->buf, res->L.allocated, st);
    return launch_lincomb2<double>((double *)res->buf, res->L, a1, (const double *)g1->buf, a2, (const double *)g2->buf, st);
  }
  if (!g2) return launch_lincomb1<float>((float *)res->buf, (float)a1, (const float *)g1->buf, res->L.allocated, st);
  return launch_lincomb2<float>((float *)res->buf, res->L, (float)a1, (const float *)g1->buf, (float)a2,
                                (const float *)g2->buf, st);
}

ocu_status ocu_grid_reduce(const ocu_grid *g, ocu_reduce_op op, double *result, ocu_stream s) {
  OCU_NOT_NULL(g, "grid");
  OCU_NOT_NULL(result, "result");
  if (op < OCU_REDUCE_MAXABS || op > OCU_REDUCE_CHECKNAN) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] reduce - bad op");
  cudaStream_t st = (cudaStream_t)s;
  // [counter | block partials | result]: the result slot starts on a 64-byte boundary
  const size_t base = ((reduce_scratch_bytes(g->L, dtype_size(g->dtype)) + 63) / 64) * 64;
  const size_t bytes = base + 64;
  char *scratch = nullptr;
  OCU_TRY(check_cuda(cudaMallocAsync((void **)&scratch, bytes, st), "cudaMallocAsync(reduce)"));
  ocu_status rs = check_cuda(cudaMemsetAsync(scratch, 0, bytes, st), "cudaMemsetAsync(reduce)");
  double *d_res = (double *)(scratch + base);
  if (rs == OCU_OK) {
    if (g->dtype == OCU_F64) rs = launch_reduce<double>(origin<double>(g), g->L, op, scratch, d_res, st);
    else rs = launch_reduce<float>(origin<float>(g), g->L, op, scratch, d_res, st);
  }
  double h = 0;
  if (rs == OCU_OK) rs = check_cuda(cudaMemcpyAsync(&h, d_res, sizeof(double), cudaMemcpyDeviceToHost, st), "reduce readback");
  cudaFreeAsync(scratch, st);
  if (rs == OCU_OK) rs = check_cuda(cudaStreamSynchronize(st), "reduce");
  if (rs == OCU_OK) *result = h;
  return rs;
}

ocu_status ocu_apply_boundary_conditions(ocu_grid *g, const ocu_bc_set *bc, double hx, double hy, double hz,
                                         ocu_bc_variant variant, ocu_stream s) {
  OCU_NOT_NULL(g, "grid");
  OCU_NOT_NULL(bc, "bc");
  cudaStream_t st = (cudaStream_t)s;
  if (variant == OCU_BC_LEVEL1) {
    if (g->dtype == OCU_F64) return launch_bc_level1<double>(origin<double>(g), g->L, *bc, hx, hy, hz, st);
    return launch_bc_level1<float>(origin<float>(g), g->L, *bc, hx, hy, hz, st);
  }
  if (variant == OCU_BC_LEVEL1_NOCORNERS) {
    if (g->dtype == OCU_F64) return launch_bc_nocorners_dev<double>(origin<double>(g), g->L, *bc, hx, hy, hz, st);
    return launch_bc_nocorners_dev<float>(origin<float>(g), g->L, *bc, hx, hy, hz, st);
  }
  return fail(OCU_ERR_INVALID_VALUE, "[ERROR] apply_boundary_conditions - unknown variant %d", (int)variant);
}

ocu_status ocu_apply_mac_boundary_conditions(ocu_grid *u, ocu_grid *v, ocu_grid *w, const ocu_bc_set *bc, double hx,
                                             double hy, double hz, ocu_stream s) {
  OCU_NOT_NULL(u, "u"); OCU_NOT_NULL(v, "v"); OCU_NOT_NULL(w, "w"); OCU_NOT_NULL(bc, "bc");
  (void)hx; (void)hy; (void)hz;
  if (!layout_match(u->L, v->L) || !layout_match(u->L, w->L))
    return fail(OCU_ERR_LAYOUT, "[ERROR] apply_3d_mac_boundary_conditions_level1 - layout mismatch");
  const int nx = u->L.nx - 1, ny = u->L.ny, nz = u->L.nz;
  if (v->L.nx != nx || v->L.ny != ny + 1 || v->L.nz != nz)
    return fail(OCU_ERR_LAYOUT, "[ERROR] apply_3d_mac_boundary_conditions_level1 - v_grid dimension mismatch");
  if (w->L.nx != nx || w->L.ny != ny || w->L.nz != nz + 1)
    return fail(OCU_ERR_LAYOUT, "[ERROR] apply_3d_mac_boundary_conditions_level1 - w_grid dimension mismatch");
  if (u->dtype != v->dtype || u->dtype != w->dtype) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] mac bc - element type mismatch");
  cudaStream_t st = (cudaStream_t)s;
  if (u->dtype == OCU_F64)
    return launch_mac_bc_level1<double>(origin<double>(u), origin<double>(v), origin<double>(w), u->L, nx, ny, nz, *bc, st);
  return launch_mac_bc_level1<float>(origin<float>(u), origin<float>(v), origin<float>(w), u->L, nx, ny, nz, *bc, st);
}

static bool same3(const ocu_grid *a, const ocu_grid *b, const ocu_grid *c) {
  return layout_match(a->L, b->L) && layout_match(a->L, c->L) && a->dtype == b->dtype && a->dtype == c->dtype;
}

ocu_status ocu_divergence(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w, ocu_grid *div, int nx, int ny,
                          int nz, double hx, double hy, double hz, ocu_stream s) {
  OCU_NOT_NULL(u, "u"); OCU_NOT_NULL(v, "v"); OCU_NOT_NULL(w, "w"); OCU_NOT_NULL(div, "divergence");
  if (!same3(u, v, w) || !layout_match(u->L, div->L) || div->dtype != u->dtype)
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_Divergence3DDevice::initialize_storage - invalid dimensions for divergence");
  cudaStream_t st = (cudaStream_t)s;
  if (u->dtype == OCU_F64)
    return launch_divergence<double>(origin<double>(u), origin<double>(v), origin<double>(w), origin<double>(div), u->L,
                                     nx, ny, nz, hx, hy, hz, st);
  return launch_divergence<float>(origin<float>(u), origin<float>(v), origin<float>(w), origin<float>(div), u->L, nx,
                                  ny, nz, hx, hy, hz, st);
}

ocu_status ocu_gradient_add(ocu_grid *u, ocu_grid *v, ocu_grid *w, const ocu_grid *phi, double coefficient, double hx,
                            double hy, double hz, ocu_stream s) {
  OCU_NOT_NULL(u, "u"); OCU_NOT_NULL(v, "v"); OCU_NOT_NULL(w, "w"); OCU_NOT_NULL(phi, "phi");
  if (!same3(u, v, w) || !layout_match(u->L, phi->L) || phi->dtype != u->dtype)
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_Gradient3DDevice::initialize_storage - invalid dimensions for phi");
  cudaStream_t st = (cudaStream_t)s;
  if (u->dtype == OCU_F64)
    return launch_gradient<double>(origin<double>(u), origin<double>(v), origin<double>(w), origin<double>(phi), u->L,
                                   phi->L.nx, phi->L.ny, phi->L.nz, hx, hy, hz, (double)coefficient, st);
  return launch_gradient<float>(origin<float>(u), origin<float>(v), origin<float>(w), origin<float>(phi), u->L, phi->L.nx,
                                phi->L.ny, phi->L.nz, hx, hy, hz, (float)coefficient, st);
}

ocu_status ocu_advect_self(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w, ocu_grid *du, ocu_grid *dv,
                           ocu_grid *dw, int nx, int ny, int nz, double hx, double hy, double hz,
                           ocu_interpolation interp, ocu_stream s) {
  OCU_NOT_NULL(u, "u"); OCU_NOT_NULL(v, "v"); OCU_NOT_NULL(w, "w");
  OCU_NOT_NULL(du, "dudt"); OCU_NOT_NULL(dv, "dvdt"); OCU_NOT_NULL(dw, "dwdt");
  if (!same3(u, v, w) || !same3(u, du, dv) || !layout_match(u->L, dw->L) || dw->dtype != u->dtype)
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_SelfAdvection3DDevice::initialize_storage - u,v,w layout mismatch");
  if (u->L.nx != nx + 1 || v->L.ny != ny + 1 || w->L.nz != nz + 1)
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_SelfAdvection3DDevice::initialize_storage - u dimensions mismatch");
  cudaStream_t st = (cudaStream_t)s;
  if (u->dtype == OCU_F64)
    return launch_advect_self<double>(origin<double>(u), origin<double>(v), origin<double>(w), origin<double>(du),
                                      origin<double>(dv), origin<double>(dw), u->L, nx, ny, nz, hx, hy, hz, interp, st);
  return launch_advect_self<float>(origin<float>(u), origin<float>(v), origin<float>(w), origin<float>(du),
                                   origin<float>(dv), origin<float>(dw), u->L, nx, ny, nz, hx, hy, hz, interp, st);
}

ocu_status ocu_advect_passive(const ocu_grid *u, const ocu_grid *v, const ocu_grid *w, const ocu_grid *phi,
                              ocu_grid *dphi, int nx, int ny, int nz, double hx, double hy, double hz,
                              ocu_interpolation interp, ocu_stream s) {
  OCU_NOT_NULL(u, "u"); OCU_NOT_NULL(v, "v"); OCU_NOT_NULL(w, "w"); OCU_NOT_NULL(phi, "phi"); OCU_NOT_NULL(dphi, "dphidt");
  if (!same3(u, v, w) || !same3(u, phi, dphi))
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_PassiveAdvection3DDevice::initialize_storage - layout mismatch");
  cudaStream_t st = (cudaStream_t)s;
  if (u->dtype == OCU_F64)
    return launch_advect_passive<double>(origin<double>(u), origin<double>(v), origin<double>(w), origin<double>(phi),
                                         origin<double>(dphi), u->L, nx, ny, nz, hx, hy, hz, interp, st);
  return launch_advect_passive<float>(origin<float>(u), origin<float>(v), origin<float>(w), origin<float>(phi),
                                      origin<float>(dphi), u->L, nx, ny, nz, hx, hy, hz, interp, st);
}

ocu_status ocu_laplacian_add(const ocu_grid *phi, ocu_grid *dphi, int nx, int ny, int nz, double hx, double hy,
                             double hz, double coefficient, ocu_stream s) {
  OCU_NOT_NULL(phi, "phi"); OCU_NOT_NULL(dphi, "dphidt");
  if (!layout_match(phi->L, dphi->L) || phi->dtype != dphi->dtype)
    return fail(OCU_ERR_LAYOUT, "[ERROR] Sol_LaplacianCentered3DDevice::initialize_storage - layout mismatch");
  cudaStream_t st = (cudaStream_t)s;
  if (phi->dtype == OCU_F64)
    return launch_laplacian<double>(origin<double>(phi), origin<double>(dphi), phi->L, nx, ny, nz, hx, hy, hz,
                                    coefficient, st);
  return launch_laplacian<float>(origin<float>(phi), origin<float>(dphi), phi->L, nx, ny, nz, hx, hy, hz,
                                 (float)coefficient, st);
}

// ---- multigrid ----------------------------------------------------------------------------
void ocu_mg_params_default(ocu_mg_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->nu1 = 2;
  p->nu2 = 2;
  p->convergence = OCU_CONVERGENCE_L2;
  p->ir_inner_cycles = 4;
}

ocu_status ocu_mg_create(ocu_mg_kind kind, const ocu_mg_params *params, ocu_mg **out) {
  OCU_NOT_NULL(out, "out");
  *out = nullptr;
  if (kind < OCU_MG_F32 || kind > OCU_MG_MIXED_WARMSTART) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_mg_create - bad kind");
  ocu_mg_params p;
  if (params) p = *params; else ocu_mg_params_default(&p);
  *out = new (std::nothrow) ocu_mg(kind, p);
  return *out ? OCU_OK : fail(OCU_ERR_ALLOC, "[ERROR] ocu_mg_create - out of host memory");
}

void ocu_mg_destroy(ocu_mg *mg) { delete mg; }

ocu_status ocu_mg_set_params(ocu_mg *mg, const ocu_mg_params *p) {
  OCU_NOT_NULL(mg, "solver"); OCU_NOT_NULL(p, "params");
  return mg->s.set_params(*p);
}

ocu_status ocu_mg_get_params(const ocu_mg *mg, ocu_mg_params *p) {
  OCU_NOT_NULL(mg, "solver"); OCU_NOT_NULL(p, "params");
  *p = mg->s.prm;
  return OCU_OK;
}

ocu_status ocu_mg_set_stream(ocu_mg *mg, ocu_stream s) {
  OCU_NOT_NULL(mg, "solver");
  mg->s.set_stream((cudaStream_t)s);
  return OCU_OK;
}

ocu_status ocu_mg_initialize_storage(ocu_mg *mg, int nx, int ny, int nz, double hx, double hy, double hz, ocu_grid *rhs) {
  OCU_NOT_NULL(mg, "solver");
  return mg->s.initialize_storage(nx, ny, nz, hx, hy, hz, rhs);
}

ocu_status ocu_mg_solve(ocu_mg *mg, double *residual, double tolerance, int max_iter) {
  OCU_NOT_NULL(mg, "solver");
  double r = 0;
  ocu_status st = mg->s.solve(&r, tolerance, max_iter);
  if (residual) *residual = r;
  return st;
}

ocu_status ocu_mg_run_vcycles(ocu_mg *mg, int count) {
  OCU_NOT_NULL(mg, "solver");
  return mg->s.run_vcycles(count);
}

ocu_status ocu_mg_run_fmg(ocu_mg *mg, int count) {
  OCU_NOT_NULL(mg, "solver");
  return mg->s.run_fmg(count);
}

ocu_grid *ocu_mg_pressure(ocu_mg *mg) { return mg ? mg->s.pressure : nullptr; }

ocu_grid *ocu_mg_level_grid(ocu_mg *mg, char which, int level) { return mg ? mg->s.level_grid(which, level) : nullptr; }

static ocu_status pick_core(ocu_mg *mg, int core, int level, CoreOps **out) {
  OCU_NOT_NULL(mg, "solver");
  if (!mg->s.initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] level operation - not initialized");
  CoreOps *c;
  if (core == 1) {
    if (mg->s.kind != OCU_MG_MIXED_IR && mg->s.kind != OCU_MG_MIXED_WARMSTART && mg->s.kind != OCU_MG_F32)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] level operation - solver has no FP32 hierarchy");
    c = &mg->s.cf;
  } else if (core == 0) {
    if (mg->s.co) c = mg->s.co->ops();
    else c = mg->s.kind == OCU_MG_F32 ? (CoreOps *)&mg->s.cf : (CoreOps *)&mg->s.cd;
  } else {
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] level operation - bad core %d", core);
  }
  if (level < 0 || level >= c->levels()) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] level operation - bad level %d", level);
  *out = c;
  return OCU_OK;
}

// core 2: the red/black split FP32 hierarchy of a refinement solver (ir_chequer.cu)
static ocu_status pick_chequer(ocu_mg *mg, int level, ChequerMG **out) {
  OCU_NOT_NULL(mg, "solver");
  if (!mg->s.initialized) return fail(OCU_ERR_NOT_INITIALIZED, "[ERROR] level operation - not initialized");
  if (!mg->s.chq) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] level operation - solver has no split FP32 hierarchy");
  if (level < 0 || level >= mg->s.chq->levels()) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] level operation - bad level %d", level);
  *out = mg->s.chq.get();
  return OCU_OK;
}

ocu_status ocu_mg_relax(ocu_mg *mg, int core, int level, int iterations, int order) {
  if (core == 2) {
    ChequerMG *q;
    OCU_TRY(pick_chequer(mg, level, &q));
    if (iterations < 0 || order < 0 || order > 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] relax - bad arguments");
    return q->relax_level(level, iterations, order == 1, mg->s.stream);
  }
  CoreOps *c;
  OCU_TRY(pick_core(mg, core, level, &c));
  if (iterations < 0 || order < 0 || order > 2) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] relax - bad arguments");
  return c->relax(level, iterations, order);
}

ocu_status ocu_mg_relax_sweep(ocu_mg *mg, int core, int level, int color) {
  if (core == 2) {
    ChequerMG *q;
    OCU_TRY(pick_chequer(mg, level, &q));
    return q->sweep_level(level, color, mg->s.stream);
  }
  CoreOps *c;
  OCU_TRY(pick_core(mg, core, level, &c));
  return c->relax_sweep(level, color & 1);
}

ocu_status ocu_mg_restrict_residuals(ocu_mg *mg, int core, int fine, int coarse, double *l2, double *linf) {
  if (core == 2) {
    ChequerMG *q;
    OCU_TRY(pick_chequer(mg, fine, &q));
    if (coarse != fine + 1 || coarse >= q->levels() || l2 || linf)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] restrict_residuals - the split hierarchy restricts into the next level, without norms");
    return q->restrict_level(fine, mg->s.stream);
  }
  CoreOps *c;
  OCU_TRY(pick_core(mg, core, fine, &c));
  if (coarse != fine && coarse != fine + 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] restrict_residuals - bad levels");
  if (coarse >= c->levels()) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] restrict_residuals - bad coarse level");
  return c->restrict_residuals(fine, coarse, l2, linf);
}

ocu_status ocu_mg_prolong(ocu_mg *mg, int core, int coarse, int fine) {
  if (core == 2) {
    ChequerMG *q;
    OCU_TRY(pick_chequer(mg, fine, &q));
    if (coarse != fine + 1 || coarse >= q->levels()) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] prolong - bad levels");
    return q->prolong_level(coarse, mg->s.stream);
  }
  CoreOps *c;
  OCU_TRY(pick_core(mg, core, fine, &c));
  if (coarse != fine + 1 || coarse >= c->levels()) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] prolong - bad levels");
  return c->prolong(coarse, fine);
}

ocu_status ocu_mg_synchronize(ocu_mg *mg) {
  OCU_NOT_NULL(mg, "solver");
  if (mg->s.co) OCU_TRY(mg->s.co->ops()->join());
  return check_cuda(cudaStreamSynchronize(mg->s.stream), "synchronize");
}

ocu_status ocu_mg_get_stats(const ocu_mg *mg, ocu_mg_stats *stats) {
  OCU_NOT_NULL(mg, "solver"); OCU_NOT_NULL(stats, "stats");
  *stats = mg->s.stats;
  return OCU_OK;
}

// ---- projection -----------------------------------------------------------------------------
ocu_status ocu_project_create_with(ocu_mg_kind kind, ocu_project **out) {
  OCU_NOT_NULL(out, "out");
  *out = nullptr;
  if (kind < OCU_MG_F32 || kind > OCU_MG_MIXED_WARMSTART)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_project_create_with - bad pressure solver kind");
  *out = new (std::nothrow) ocu_project();
  if (!*out) return fail(OCU_ERR_ALLOC, "[ERROR] ocu_project_create - out of host memory");
  (*out)->s.dtype = kind == OCU_MG_F32 ? OCU_F32 : OCU_F64;
  (*out)->s.mg_kind = kind;
  return OCU_OK;
}

ocu_status ocu_project_create_fields(ocu_dtype fields, ocu_mg_kind kind, ocu_project **out) {
  OCU_NOT_NULL(out, "out");
  *out = nullptr;
  if (fields == OCU_F32 && kind == OCU_MG_MIXED_IR) {
    *out = new (std::nothrow) ocu_project();
    if (!*out) return fail(OCU_ERR_ALLOC, "[ERROR] ocu_project_create - out of host memory");
    (*out)->s.dtype = OCU_F32;
    (*out)->s.mg_kind = kind;
    return OCU_OK;
  }
  if ((fields == OCU_F32) != (kind == OCU_MG_F32))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_project_create_fields - unsupported field / pressure combination");
  return ocu_project_create_with(kind, out);
}

ocu_status ocu_project_create(ocu_dtype dtype, ocu_project **out) {
  if (dtype != OCU_F32 && dtype != OCU_F64) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_project_create - bad dtype");
  return ocu_project_create_with(dtype == OCU_F64 ? OCU_MG_F64 : OCU_MG_F32, out);
}

void ocu_project_destroy(ocu_project *p) { delete p; }

ocu_status ocu_project_set_stream(ocu_project *p, ocu_stream s) {
  OCU_NOT_NULL(p, "projection");
  p->s.set_stream((cudaStream_t)s);
  return OCU_OK;
}

ocu_status ocu_project_initialize_storage(ocu_project *p, int nx, int ny, int nz, double hx, double hy, double hz,
                                          ocu_grid *u, ocu_grid *v, ocu_grid *w, const ocu_bc_set *bc) {
  OCU_NOT_NULL(p, "projection"); OCU_NOT_NULL(bc, "bc");
  return p->s.initialize_storage(nx, ny, nz, hx, hy, hz, u, v, w, *bc);
}

ocu_status ocu_project_solve(ocu_project *p, double tolerance) {
  OCU_NOT_NULL(p, "projection");
  ocu_status st = p->s.solve(tolerance);
  if (st == OCU_OK || st == OCU_ERR_NOT_CONVERGED) {
    ocu_status s2 = check_cuda(cudaStreamSynchronize(p->s.stream), "Sol_ProjectDivergence3DDevice::solve");
    if (s2 != OCU_OK) return s2;
  }
  return st;
}

ocu_status ocu_project_solve_divergence_only(ocu_project *p) {
  OCU_NOT_NULL(p, "projection");
  return p->s.solve_divergence_only();
}

ocu_grid *ocu_project_divergence(ocu_project *p) { return p ? p->s.divergence : nullptr; }
ocu_mg *ocu_project_pressure_solver(ocu_project *p) { return p ? p->s.mg : nullptr; }

// ---- Navier-Stokes ----------------------------------------------------------------------------
void ocu_ns_params_default(ocu_ns_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->advection_scheme = OCU_IT_FIRST_ORDER_UPWIND;
  p->max_divergence = 1e-5;
  p->cfl_factor = 1;
  p->gravity = -9.8;
  p->bouyancy = 1;
  p->time_step = OCU_TS_FORWARD_EULER;
  p->vertical_direction = OCU_DIR_YPOS;
}

ocu_status ocu_ns_init_layout(int nx, int ny, int nz, char which, ocu_layout *out) {
  OCU_NOT_NULL(out, "layout");
  return ns_init_layout(nx, ny, nz, which, out);
}

ocu_status ocu_ns_create(ocu_dtype dtype, ocu_ns **out) {
  OCU_NOT_NULL(out, "out");
  *out = new (std::nothrow) ocu_ns();
  if (!*out) return fail(OCU_ERR_ALLOC, "[ERROR] ocu_ns_create - out of host memory");
  (*out)->s.dtype = dtype;
  return OCU_OK;
}

void ocu_ns_destroy(ocu_ns *ns) { delete ns; }

ocu_status ocu_ns_set_stream(ocu_ns *ns, ocu_stream s) {
  OCU_NOT_NULL(ns, "equation");
  ns->s.set_stream((cudaStream_t)s);
  return OCU_OK;
}

ocu_status ocu_ns_set_parameters(ocu_ns *ns, const ocu_ns_params *p, const void *iu, const void *iv, const void *iw,
                                 const void *it) {
  OCU_NOT_NULL(ns, "equation"); OCU_NOT_NULL(p, "params");
  OCU_NOT_NULL(iu, "init_u"); OCU_NOT_NULL(iv, "init_v"); OCU_NOT_NULL(iw, "init_w"); OCU_NOT_NULL(it, "init_temp");
  if (ns->s.initialized) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] set_parameters - already initialized");
  return ns->s.set_parameters(*p, iu, iv, iw, it);
}

ocu_status ocu_ns_get_max_stable_timestep(ocu_ns *ns, double *dt) {
  OCU_NOT_NULL(ns, "equation"); OCU_NOT_NULL(dt, "dt");
  return ns->s.get_max_stable_timestep(dt);
}

ocu_status ocu_ns_advance_one_step(ocu_ns *ns, double dt) {
  OCU_NOT_NULL(ns, "equation");
  ocu_status st = ns->s.advance_one_step(dt);
  if (st == OCU_OK) st = check_cuda(cudaStreamSynchronize(ns->s.stream), "advance_one_step");
  return st;
}

ocu_status ocu_ns_advance(ocu_ns *ns, double dt) {
  OCU_NOT_NULL(ns, "equation");
  ocu_status st = ns->s.advance(dt);
  if (st == OCU_OK) st = check_cuda(cudaStreamSynchronize(ns->s.stream), "advance");
  return st;
}

ocu_grid *ocu_ns_grid(ocu_ns *ns, char which) { return ns ? ns->s.grid(which) : nullptr; }
int ocu_ns_num_steps(const ocu_ns *ns) { return ns ? ns->s.num_steps : 0; }

}  // extern "C"
