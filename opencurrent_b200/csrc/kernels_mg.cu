// Multigrid level kernels: red-black SOR sweeps, coarsest-level solve, residual, restriction,
// prolongation, and the FP32<->FP64 transfers of the iterative-refinement solver.
//
// Arithmetic follows the reference kernels operation by operation (file:line at each kernel);
// the library is built with --fmad=false, so results are bit-identical to the CPU oracle.
#include "bc_device.cuh"
#include "mg_fused.h"
#include "ocu_internal.h"

namespace ocub {

// Coefficients of one colour sweep, already rounded to T the way the reference launcher rounds
// them (sol_mgpressure3ddevf.cu:390-393 for float, sol_mgpressure3ddevd.cu:1262-1268 for
// double).
template <typename T>
struct RelaxCoef {
  T omega, hsq, fx, fy, fz, ld;    // hsq = (T)(h*h) for float, (-h)*h for double
  T xp, xn, yp, yn, zp, zn;        // bc_diag_mod per face
};

template <typename T>
RelaxCoef<T> make_relax_coef(const RelaxParams &p) {
  RelaxCoef<T> c;
  c.omega = (T)p.omega;
  c.hsq = sizeof(T) == 4 ? (T)(p.h * p.h) : (T)(-p.h * p.h);
  c.fx = (T)p.fx; c.fy = (T)p.fy; c.fz = (T)p.fz;
  c.ld = (T)(2 * p.fx + 2 * p.fy + 2 * p.fz);
  c.xp = (T)bc_diag_mod(p.bc.xpos, p.fx); c.xn = (T)bc_diag_mod(p.bc.xneg, p.fx);
  c.yp = (T)bc_diag_mod(p.bc.ypos, p.fy); c.yn = (T)bc_diag_mod(p.bc.yneg, p.fy);
  c.zp = (T)bc_diag_mod(p.bc.zpos, p.fz); c.zn = (T)bc_diag_mod(p.bc.zneg, p.fz);
  return c;
}

// One colour of red-black SOR, in place: cells with (i+j+k+colour) even, k = 2t + parity for
// t < nz/2.  Float: Sol_MultigridPressure3DDeviceF_relax (devf.cu:200-252).  Double:
// ..._relax_DIAG (devd.cu:542-599), whose x/y diagonal comes from a 2D table built once at
// initialize_storage (sol_mgpressure3ddev.cu:27-43).
template <typename T>
__global__ void __launch_bounds__(256) k_relax_color(T *__restrict__ u, const T *__restrict__ b, long long xs,
                                                     long long ys, int nx, int ny, int nz, int color,
                                                     RelaxCoef<T> c, const T *__restrict__ diag) {
  pdl_entry();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= nx || j >= ny || t >= nz / 2) return;
  const int k = 2 * t + ((i + j + color) & 1);
  const long long id = (long long)i * xs + (long long)j * ys + k;
  const T uc = u[id];
  T res;
  T dg;
  if (sizeof(T) == 4) {
    const T bv = b[id];
    res = (-c.hsq * bv - c.ld * uc);
    res += c.fz * (u[id - 1] + u[id + 1]);
    res += c.fy * (u[id - ys] + u[id + ys]);
    res += c.fx * (u[id - xs] + u[id + xs]);
    dg = c.ld;
    if (i == nx - 1) dg += c.xp;
    if (i == 0) dg += c.xn;
    if (j == ny - 1) dg += c.yp;
    if (j == 0) dg += c.yn;
    if (k == nz - 1) dg += c.zp;
    if (k == 0) dg += c.zn;
  } else {
    res = -c.ld * uc;
    res += c.fz * (u[id - 1] + u[id + 1]);
    res += c.fy * (u[id - ys] + u[id + ys]);
    res += c.fx * (u[id - xs] + u[id + xs]);
    res += c.hsq * b[id];
    dg = diag[(long long)i * ny + j];
    if (k == nz - 1) dg += c.zp;
    if (k == 0) dg += c.zn;
  }
  u[id] = uc + c.omega * res / dg;
}

template <typename T>
ocu_status launch_relax_color(T *u, const T *b, const ocu_layout &L, const T *diag, int color,
                              const RelaxParams &p, cudaStream_t s) {
  const RelaxCoef<T> c = make_relax_coef<T>(p);
  const int half = L.nz / 2;
  if (half == 0) return OCU_OK;
  dim3 block(half >= 32 ? 32 : (half >= 16 ? 16 : (half >= 8 ? 8 : 4)), 4, 2);
  block.y = 256 / (block.x * block.z) > 8 ? 8 : 256 / (block.x * block.z);
  dim3 grid((half + block.x - 1) / block.x, (L.ny + block.y - 1) / block.y, (L.nx + block.z - 1) / block.z);
  launch_pdl(k_relax_color<T>, grid, block, 0, s, u, b, L.xstride, L.ystride, L.nx, L.ny, L.nz, color, c, diag);
  return check_launch("k_relax_color");
}

// 2D table of the diagonal plus x/y boundary modifiers (sol_mgpressure3ddev.cu:27-43).
template <typename T>
__global__ void k_init_diag(T *grid, int nx, int ny, T ld, T xp, T xn, T yp, T yn) {
  pdl_entry();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < nx && j < ny) {
    T d = ld;
    if (i == nx - 1) d += xp;
    if (i == 0) d += xn;
    if (j == ny - 1) d += yp;
    if (j == 0) d += yn;
    grid[(long long)i * ny + j] = d;
  }
}

template <typename T>
ocu_status launch_init_diag(T *diag, int nx, int ny, const RelaxParams &p, cudaStream_t s) {
  const RelaxCoef<T> c = make_relax_coef<T>(p);
  dim3 block(16, 16), grid((nx + 15) / 16, (ny + 15) / 16);
  launch_pdl(k_init_diag<T>, grid, block, 0, s, diag, nx, ny, c.ld, c.xp, c.xn, c.yp, c.yn);
  return check_launch("k_init_diag");
}

// ------------------------------------------------------------------------------------------
// Coarsest level.  The reference copies u and b to the host, runs do_cpu_solve with host ghost
// fills after every colour, copies back and re-applies the device ghost fill
// (sol_mgpressure3ddev.cu:82-188).  Here the same sequence runs as ONE single-CTA kernel
// (coarse_relax_block in mg_fused.h).  No PCIe round trip.
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(512) k_coarse_relax(T *u, const T *b, long long xs, long long ys, int nx, int ny,
                                                      int nz, int iterations, int order, CoarseCoef<T> c,
                                                      BCDev bc, T hx, T hy, T hz) {
  pdl_entry();
  coarse_relax_block<T>(u, b, xs, ys, nx, ny, nz, iterations, order, c, bc, hx, hy, hz);
}

// The same with u and b staged in shared memory (small coarsest levels): the ~4 phases per
// iteration then wait on shared-memory latency instead of global-memory round trips.
template <typename T>
__global__ void __launch_bounds__(512) k_coarse_relax_smem(T *u, const T *b, long long shift, long long n,
                                                           long long xs, long long ys, int nx, int ny, int nz,
                                                           int iterations, int order, CoarseCoef<T> c, BCDev bc,
                                                           T hx, T hy, T hz) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char coarse_smem[];
  T *su = reinterpret_cast<T *>(coarse_smem);
  T *sb = su + n;
  T *ub = u - shift;
  const T *bb = b - shift;
  for (long long q = threadIdx.x; q < n; q += blockDim.x) {
    su[q] = ub[q];
    sb[q] = bb[q];
  }
  __syncthreads();
  coarse_relax_block<T>(su + shift, sb + shift, xs, ys, nx, ny, nz, iterations, order, c, bc, hx, hy, hz);
  for (long long q = threadIdx.x; q < n; q += blockDim.x) ub[q] = su[q];
}

template <typename T>
ocu_status launch_coarse_relax(T *u, const T *b, const ocu_layout &L, int iterations, int order,
                               const RelaxParams &p, double hx, double hy, double hz,
                               cudaStream_t s) {
  if (!bc_check_scalar(p.bc))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] relax_on_host - invalid boundary condition types");
  const CoarseCoef<T> c = make_coarse_coef<T>(p);
  // RO_SYMMETRIC needs an even iteration count of at least 4 (sol_mgpressure3ddev.cu:159-163)
  if (order == 2) {
    if (iterations % 2 == 1) iterations++;
    if (iterations < 4) iterations = 4;
  }
  const size_t bytes = 2 * sizeof(T) * (size_t)L.allocated;
  if (bytes <= 48 * 1024) {
    launch_pdl(k_coarse_relax_smem<T>, 1, 512, bytes, s, u, b, L.shift, L.allocated, L.xstride, L.ystride, L.nx, L.ny,
               L.nz, iterations, order, c, to_dev(p.bc), (T)hx, (T)hy, (T)hz);
    return check_launch("k_coarse_relax_smem");
  }
  launch_pdl(k_coarse_relax<T>, 1, 512, 0, s, u, b, L.xstride, L.ystride, L.nx, L.ny, L.nz, iterations, order, c,
             to_dev(p.bc), (T)hx, (T)hy, (T)hz);
  return check_launch("k_coarse_relax");
}

// ------------------------------------------------------------------------------------------
// residual r = b - L u (devf.cu:68-90, devd.cu:94-114; coefficients devf.cu:420-427)
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_residual(const T *__restrict__ u, const T *__restrict__ b, T *__restrict__ r,
                                                  long long xs, long long ys, int nx, int ny, int nz, T fxh, T fyh,
                                                  T fzh, T dg) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= nz || j >= ny || i >= nx) return;
  const long long id = (long long)i * xs + (long long)j * ys + k;
  r[id] = b[id] - (fzh * (u[id - 1] + u[id + 1]) + fyh * (u[id - ys] + u[id + ys]) +
                   fxh * (u[id - xs] + u[id + xs]) - dg * u[id]);
}

template <typename T>
ocu_status launch_residual(const T *u, const T *b, T *r, const ocu_layout &L, double h,
                           double fx, double fy, double fz, cudaStream_t s) {
  dim3 block(L.nz >= 64 ? 64 : 32, L.nz >= 64 ? 4 : 8);
  dim3 grid((L.nz + block.x - 1) / block.x, (L.ny + block.y - 1) / block.y, L.nx);
  launch_pdl(k_residual<T>, grid, block, 0, s, u, b, r, L.xstride, L.ystride, L.nx, L.ny, L.nz, (T)(fx / (h * h)),
             (T)(fy / (h * h)), (T)(fz / (h * h)), (T)(2 * (fx + fy + fz) / (h * h)));
  return check_launch("k_residual");
}

// restrict: b_c = 1/8 * sum of the 8 children, in the reference's summation order
// (devf.cu:38-65).
template <typename T>
__global__ void __launch_bounds__(256) k_restrict(const T *__restrict__ r, long long rxs, long long rys,
                                                  T *__restrict__ bc_, long long bxs, long long bys, int bnx,
                                                  int bny, int bnz) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= bnz || j >= bny || i >= bnx) return;
  const long long ri = (long long)(2 * i) * rxs + (long long)(2 * j) * rys + 2 * k;
  bc_[(long long)i * bxs + (long long)j * bys + k] =
      (T)0.125 * (r[ri] + r[ri + 1] + r[ri + rys] + r[ri + 1 + rys] + r[ri + rxs] + r[ri + 1 + rxs] +
                  r[ri + rys + rxs] + r[ri + 1 + rys + rxs]);
}

template <typename T>
ocu_status launch_restrict(const T *r, const ocu_layout &Lf, T *bc_, const ocu_layout &Lc,
                           cudaStream_t s) {
  dim3 block(Lc.nz >= 32 ? 32 : 16, 8);
  dim3 grid((Lc.nz + block.x - 1) / block.x, (Lc.ny + block.y - 1) / block.y, Lc.nx);
  launch_pdl(k_restrict<T>, grid, block, 0, s, r, Lf.xstride, Lf.ystride, bc_, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny,
             Lc.nz);
  return check_launch("k_restrict");
}

// Trilinear prolongation + correction (devf.cu:94-197, devd.cu:118-223): one thread per coarse
// cell updates its 8 children.  The child at -xstride takes its 1/64 corner from (+1,+1,+1),
// exactly as the reference does.
template <typename T>
__global__ void __launch_bounds__(256) k_prolong(const T *__restrict__ uc, long long cx, long long cy, int cnx,
                                                 int cny, int cnz, T *__restrict__ uf, long long fxs,
                                                 long long fys) {
  pdl_entry();
  const int kc = blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  const int ic = blockIdx.z;
  if (kc >= cnz || jc >= cny || ic >= cnx) return;
  const T w1 = (T)0.421875, w2 = (T)0.140625, w3 = (T)0.046875, w4 = (T)0.015625;
  const long long tc = (long long)ic * cx + (long long)jc * cy + kc;
  const long long f = (long long)(2 * ic + 1) * fxs + (long long)(2 * jc + 1) * fys + (2 * kc + 1);
  const T c000 = uc[tc];
  const T cp00 = uc[tc + cx], c0p0 = uc[tc + cy], cpp0 = uc[tc + cx + cy];
  const T c00p = uc[tc + 1], cp0p = uc[tc + cx + 1], c0pp = uc[tc + cy + 1], cppp = uc[tc + cx + cy + 1];
  const T cm00 = uc[tc - cx], c0m0 = uc[tc - cy], cmm0 = uc[tc - cx - cy], c00m = uc[tc - 1];
  const T cm0m = uc[tc - cx - 1], c0mm = uc[tc - cy - 1], cmmm = uc[tc - cx - cy - 1];
  const T cmp0 = uc[tc - cx + cy], cm0p = uc[tc - cx + 1], cpm0 = uc[tc + cx - cy];
  const T c0mp = uc[tc - cy + 1], cp0m = uc[tc + cx - 1], c0pm = uc[tc + cy - 1];
  const T cpmm = uc[tc + cx - cy - 1], cmpm = uc[tc - cx + cy - 1], cmmp = uc[tc - cx - cy + 1];
  const T cppm = uc[tc + cx + cy - 1], cpmp = uc[tc + cx - cy + 1];
  uf[f] = uf[f] + w1 * c000 + w2 * (cp00 + c0p0 + c00p) + w3 * (cpp0 + cp0p + c0pp) + w4 * cppp;
  uf[f - fxs] = uf[f - fxs] + w1 * c000 + w2 * (cm00 + c0p0 + c00p) + w3 * (cmp0 + cm0p + c0pp) + w4 * cppp;
  uf[f - fys] = uf[f - fys] + w1 * c000 + w2 * (cp00 + c0m0 + c00p) + w3 * (cpm0 + cp0p + c0mp) + w4 * cpmp;
  uf[f - 1] = uf[f - 1] + w1 * c000 + w2 * (cp00 + c0p0 + c00m) + w3 * (cpp0 + cp0m + c0pm) + w4 * cppm;
  uf[f - fxs - fys] = uf[f - fxs - fys] + w1 * c000 + w2 * (cm00 + c0m0 + c00p) + w3 * (cmm0 + cm0p + c0mp) + w4 * cmmp;
  uf[f - fxs - 1] = uf[f - fxs - 1] + w1 * c000 + w2 * (cm00 + c0p0 + c00m) + w3 * (cmp0 + cm0m + c0pm) + w4 * cmpm;
  uf[f - fys - 1] = uf[f - fys - 1] + w1 * c000 + w2 * (cp00 + c0m0 + c00m) + w3 * (cpm0 + cp0m + c0mm) + w4 * cpmm;
  uf[f - fxs - fys - 1] = uf[f - fxs - fys - 1] + w1 * c000 + w2 * (cm00 + c0m0 + c00m) + w3 * (cmm0 + cm0m + c0mm) + w4 * cmmm;
}

template <typename T>
ocu_status launch_prolong(const T *uc, const ocu_layout &Lc, T *uf, const ocu_layout &Lf,
                          cudaStream_t s) {
  dim3 block(Lc.nz >= 32 ? 32 : 16, 8);
  dim3 grid((Lc.nz + block.x - 1) / block.x, (Lc.ny + block.y - 1) / block.y, Lc.nx);
  launch_pdl(k_prolong<T>, grid, block, 0, s, uc, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, uf, Lf.xstride, Lf.ystride);
  return check_launch("k_prolong");
}

// ------------------------------------------------------------------------------------------
// Iterative refinement transfers (no reference counterpart).
// ------------------------------------------------------------------------------------------
__global__ void k_downcast_interior(const double *__restrict__ r, float *__restrict__ b, long long xs, long long ys,
                                    int nx, int ny, int nz) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= nz || j >= ny || i >= nx) return;
  const long long id = (long long)i * xs + (long long)j * ys + k;
  b[id] = (float)r[id];
}

__global__ void k_add_correction(double *__restrict__ x, const float *__restrict__ e, long long xs, long long ys,
                                 int nx, int ny, int nz) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= nz || j >= ny || i >= nx) return;
  const long long id = (long long)i * xs + (long long)j * ys + k;
  x[id] = x[id] + (double)e[id];
}

// The same, two cells per thread (double2 / float2; nz even, rows on 2-element boundaries).
__global__ void k_add_correction2(double *__restrict__ x, const float *__restrict__ e, long long xs, long long ys,
                                  int nx, int ny, int nz) {
  pdl_entry();
  const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= nz || j >= ny || i >= nx) return;
  const long long id = (long long)i * xs + (long long)j * ys + k;
  double2 xv = *reinterpret_cast<const double2 *>(x + id);
  const float2 ev = *reinterpret_cast<const float2 *>(e + id);
  xv.x = xv.x + (double)ev.x;
  xv.y = xv.y + (double)ev.y;
  *reinterpret_cast<double2 *>(x + id) = xv;
}

ocu_status launch_downcast_interior(const double *r, float *b32, const ocu_layout &L,
                                    cudaStream_t s) {
  dim3 block(64, 4), grid((L.nz + 63) / 64, (L.ny + 3) / 4, L.nx);
  launch_pdl(k_downcast_interior, grid, block, 0, s, r, b32, L.xstride, L.ystride, L.nx, L.ny, L.nz);
  return check_launch("k_downcast_interior");
}

ocu_status launch_add_correction(double *x, const float *e, const ocu_layout &L,
                                 cudaStream_t s) {
  if (L.nz % 2 == 0 && L.shift % 2 == 0 && L.xstride % 2 == 0 && L.ystride % 2 == 0) {
    dim3 block(64, 4), grid((L.nz / 2 + 63) / 64, (L.ny + 3) / 4, L.nx);
    launch_pdl(k_add_correction2, grid, block, 0, s, x, e, L.xstride, L.ystride, L.nx, L.ny, L.nz);
    return check_launch("k_add_correction2");
  }
  dim3 block(64, 4), grid((L.nz + 63) / 64, (L.ny + 3) / 4, L.nx);
  launch_pdl(k_add_correction, grid, block, 0, s, x, e, L.xstride, L.ystride, L.nx, L.ny, L.nz);
  return check_launch("k_add_correction");
}

#define INST(T)                                                                                          \
  template ocu_status launch_relax_color<T>(T *, const T *, const ocu_layout &, const T *, int,          \
                                            const RelaxParams &, cudaStream_t);                          \
  template ocu_status launch_init_diag<T>(T *, int, int, const RelaxParams &, cudaStream_t);             \
  template ocu_status launch_coarse_relax<T>(T *, const T *, const ocu_layout &, int, int,               \
                                             const RelaxParams &, double, double, double, cudaStream_t); \
  template ocu_status launch_residual<T>(const T *, const T *, T *, const ocu_layout &, double, double,   \
                                         double, double, cudaStream_t);                                  \
  template ocu_status launch_restrict<T>(const T *, const ocu_layout &, T *, const ocu_layout &,         \
                                         cudaStream_t);                                                  \
  template ocu_status launch_prolong<T>(const T *, const ocu_layout &, T *, const ocu_layout &, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace ocub
