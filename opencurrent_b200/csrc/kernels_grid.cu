// Grid kernels: ghost fills, clear/convert/axpy and deterministic reductions.
//
// All arithmetic reproduces the reference expression order; the library is compiled with
// --fmad=false so every product and sum is rounded exactly as written.
#include <cfloat>
#include <cstdint>

#include "bc_device.cuh"
#include "ocu_internal.h"

namespace ocub {

template <typename T>
__global__ void __launch_bounds__(256) k_bc_level1(Level1Compose<T> c, long long nzreg, long long nyreg,
                                                   long long nxreg) {
  pdl_entry();
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  if (t < nzreg) {  // z faces: side, i in [-1,nx], j in [-1,ny]
    const long long per = (long long)(nx + 2) * (ny + 2);
    const int side = (int)(t / per);
    const long long r = t - side * per;
    const int i = (int)(r / (ny + 2)) - 1, j = (int)(r % (ny + 2)) - 1;
    const int k = side ? nz : -1;
    if (Level1Compose<T>::writes(c.bc.ty(side ? FZ_POS : FZ_NEG)))
      c.p[(long long)i * c.xs + (long long)j * c.ys + k] = c.az(i, j, k);
    return;
  }
  t -= nzreg;
  if (t < nyreg) {  // y faces: side, i in [-1,nx], k in [0,nz)
    const long long per = (long long)(nx + 2) * nz;
    const int side = (int)(t / per);
    const long long r = t - side * per;
    const int i = (int)(r / nz) - 1, k = (int)(r % nz);
    const int j = side ? ny : -1;
    if (Level1Compose<T>::writes(c.bc.ty(side ? FY_POS : FY_NEG)))
      c.p[(long long)i * c.xs + (long long)j * c.ys + k] = c.ay(i, j, k);
    return;
  }
  t -= nyreg;
  if (t < nxreg) {  // x faces: side, j in [0,ny), k in [0,nz)
    const long long per = (long long)ny * nz;
    const int side = (int)(t / per);
    const long long r = t - side * per;
    const int j = (int)(r / nz), k = (int)(r % nz);
    const int i = side ? nx : -1;
    if (Level1Compose<T>::writes(c.bc.ty(side ? FX_POS : FX_NEG)))
      c.p[(long long)i * c.xs + (long long)j * c.ys + k] = c.ax(i, j, k);
  }
}

template <typename T>
ocu_status launch_bc_level1(T *origin, const ocu_layout &L, const ocu_bc_set &bc, double hx,
                            double hy, double hz, cudaStream_t s) {
  if (!bc_check_scalar(bc))
    return fail(OCU_ERR_INVALID_VALUE,
                "[ERROR] apply_3d_boundary_conditions_level1 - invalid boundary condition types");
  if (L.gx < 1 || L.gy < 1 || L.gz < 1)
    return fail(OCU_ERR_LAYOUT, "[ERROR] apply_3d_boundary_conditions_level1 - must have at least 1 ghost point");
  Level1Compose<T> c;
  c.p = origin;
  c.xs = L.xstride;
  c.ys = L.ystride;
  c.nx = L.nx; c.ny = L.ny; c.nz = L.nz;
  c.bc = to_dev(bc);
  c.hx = (T)hx; c.hy = (T)hy; c.hz = (T)hz;
  const long long nzreg = 2LL * (L.nx + 2) * (L.ny + 2);
  const long long nyreg = 2LL * (L.nx + 2) * L.nz;
  const long long nxreg = 2LL * L.ny * L.nz;
  const long long total = nzreg + nyreg + nxreg;
  const int threads = 256;
  const unsigned blocks = (unsigned)((total + threads - 1) / threads);
  launch_pdl(k_bc_level1<T>, blocks, threads, 0, s, c, nzreg, nyreg, nxreg);
  return check_launch("k_bc_level1");
}

// ------------------------------------------------------------------------------------------
// Faces-only fill (kernel_apply_3d_boundary_conditions_level1_nocorners,
// grid3dboundary.cu:28-119): Dirichlet is evaluated in double, -phi + 2.0*(T)value.
// ------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T nocorner_rule(const BCDev &bc, int f, T src, T h, bool neg) {
  const int t = bc.ty(f);
  if (t == OCU_BC_DIRICHELET) return (T)((double)(-src) + 2.0 * (double)(T)bc.val(f));
  if (t == OCU_BC_NEUMANN) return neg ? src - h * (T)bc.val(f) : src + h * (T)bc.val(f);
  return src;  // periodic: the caller passed the wrapped source
}

template <typename T>
__global__ void __launch_bounds__(256) k_bc_nocorners(T *p, long long xs, long long ys, int nx, int ny, int nz,
                                                      BCDev bc, T hx, T hy, T hz) {
  pdl_entry();
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long zreg = 2LL * nx * ny, yreg = 2LL * nx * nz, xreg = 2LL * ny * nz;
  auto at = [&](int i, int j, int k) -> T & { return p[(long long)i * xs + (long long)j * ys + k]; };
  if (t < zreg) {
    const int side = (int)(t / ((long long)nx * ny));
    const long long r = t - side * (long long)nx * ny;
    const int i = (int)(r / ny), j = (int)(r % ny);
    const int f = side ? FZ_POS : FZ_NEG;
    const int ty = bc.ty(f);
    if (ty == OCU_BC_PERIODIC) at(i, j, side ? nz : -1) = at(i, j, side ? 0 : nz - 1);
    else if (ty == OCU_BC_DIRICHELET || ty == OCU_BC_NEUMANN)
      at(i, j, side ? nz : -1) = nocorner_rule<T>(bc, f, at(i, j, side ? nz - 1 : 0), hz, !side);
    return;
  }
  t -= zreg;
  if (t < yreg) {
    const int side = (int)(t / ((long long)nx * nz));
    const long long r = t - side * (long long)nx * nz;
    const int i = (int)(r / nz), k = (int)(r % nz);
    const int f = side ? FY_POS : FY_NEG;
    const int ty = bc.ty(f);
    if (ty == OCU_BC_PERIODIC) at(i, side ? ny : -1, k) = at(i, side ? 0 : ny - 1, k);
    else if (ty == OCU_BC_DIRICHELET || ty == OCU_BC_NEUMANN)
      at(i, side ? ny : -1, k) = nocorner_rule<T>(bc, f, at(i, side ? ny - 1 : 0, k), hy, !side);
    return;
  }
  t -= yreg;
  if (t < xreg) {
    const int side = (int)(t / ((long long)ny * nz));
    const long long r = t - side * (long long)ny * nz;
    const int j = (int)(r / nz), k = (int)(r % nz);
    const int f = side ? FX_POS : FX_NEG;
    const int ty = bc.ty(f);
    if (ty == OCU_BC_PERIODIC) at(side ? nx : -1, j, k) = at(side ? 0 : nx - 1, j, k);
    else if (ty == OCU_BC_DIRICHELET || ty == OCU_BC_NEUMANN)
      at(side ? nx : -1, j, k) = nocorner_rule<T>(bc, f, at(side ? nx - 1 : 0, j, k), hx, !side);
  }
}

template <typename T>
ocu_status launch_bc_nocorners_dev(T *origin, const ocu_layout &L, const ocu_bc_set &bc,
                                   double hx, double hy, double hz, cudaStream_t s) {
  if (!bc_check_scalar(bc))
    return fail(OCU_ERR_INVALID_VALUE,
                "[ERROR] apply_3d_boundary_conditions_level1_nocorners - invalid boundary condition types");
  if (L.gx < 1 || L.gy < 1 || L.gz < 1)
    return fail(OCU_ERR_LAYOUT, "[ERROR] apply_3d_boundary_conditions_level1_nocorners - must have at least 1 ghost point");
  const long long total = 2LL * L.nx * L.ny + 2LL * L.nx * L.nz + 2LL * L.ny * L.nz;
  const unsigned blocks = (unsigned)((total + 255) / 256);
  launch_pdl(k_bc_nocorners<T>, blocks, 256, 0, s, origin, L.xstride, L.ystride, L.nx, L.ny, L.nz, to_dev(bc), (T)hx,
             (T)hy, (T)hz);
  return check_launch("k_bc_nocorners");
}

// ------------------------------------------------------------------------------------------
// MAC velocity ghosts (kernel_apply_3d_mac_boundary_conditions_level1_{x,y,z},
// grid3dboundary.cu:551-714): three ordered passes; the later passes read faces the earlier
// ones wrote, so they stay separate launches.
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_mac_bc_x(T *u, T *v, T *w, BCDev bc, long long xs, long long ys, int nx, int ny, int nz) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= ny || k >= nz) return;
  auto I = [&](int i) { return (long long)i * xs + (long long)j * ys + k; };
  if (bc.ty(FX_NEG) == OCU_BC_PERIODIC) {
    u[I(-1)] = u[I(nx - 1)];
    v[I(-1)] = v[I(nx - 1)];
    w[I(-1)] = w[I(nx - 1)];
  } else if (bc.ty(FX_NEG) == OCU_BC_FORCED_INFLOW_VARIABLE_SLIP) {
    const float f = 1.0f - 2.0f * bc.auxv(FX_NEG);
    u[I(-1)] = (T)bc.val(FX_NEG);
    u[I(0)] = (T)bc.val(FX_NEG);
    v[I(-1)] = v[I(0)] * (T)f;
    w[I(-1)] = w[I(0)] * (T)f;
  }
  if (bc.ty(FX_POS) == OCU_BC_PERIODIC) {
    u[I(nx)] = u[I(0)];
    u[I(nx + 1)] = u[I(1)];
    v[I(nx)] = v[I(0)];
    w[I(nx)] = w[I(0)];
  } else if (bc.ty(FX_POS) == OCU_BC_FORCED_INFLOW_VARIABLE_SLIP) {
    const float f = 1.0f - 2.0f * bc.auxv(FX_POS);
    u[I(nx)] = (T)bc.val(FX_POS);
    u[I(nx + 1)] = (T)bc.val(FX_POS);
    v[I(nx)] = v[I(nx - 1)] * (T)f;
    w[I(nx)] = w[I(nx - 1)] * (T)f;
  }
}

template <typename T>
__global__ void k_mac_bc_y(T *u, T *v, T *w, BCDev bc, long long xs, long long ys, int nx, int ny, int nz) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(blockIdx.y * blockDim.y + threadIdx.y) - 1;
  if (i > nx || k >= nz) return;
  auto J = [&](int j) { return (long long)i * xs + (long long)j * ys + k; };
  if (bc.ty(FY_NEG) == OCU_BC_PERIODIC) {
    v[J(-1)] = v[J(ny - 1)];
    u[J(-1)] = u[J(ny - 1)];
    w[J(-1)] = w[J(ny - 1)];
  } else if (bc.ty(FY_NEG) == OCU_BC_FORCED_INFLOW_VARIABLE_SLIP) {
    const float f = 1.0f - 2.0f * bc.auxv(FY_NEG);
    v[J(-1)] = (T)bc.val(FY_NEG);
    v[J(0)] = (T)bc.val(FY_NEG);
    u[J(-1)] = u[J(0)] * (T)f;
    w[J(-1)] = w[J(0)] * (T)f;
  }
  if (bc.ty(FY_POS) == OCU_BC_PERIODIC) {
    v[J(ny)] = v[J(0)];
    v[J(ny + 1)] = v[J(1)];
    u[J(ny)] = u[J(0)];
    w[J(ny)] = w[J(0)];
  } else if (bc.ty(FY_POS) == OCU_BC_FORCED_INFLOW_VARIABLE_SLIP) {
    const float f = 1.0f - 2.0f * bc.auxv(FY_POS);
    v[J(ny)] = (T)bc.val(FY_POS);
    v[J(ny + 1)] = (T)bc.val(FY_POS);
    u[J(ny)] = u[J(ny - 1)] * (T)f;
    w[J(ny)] = w[J(ny - 1)] * (T)f;
  }
}

template <typename T>
__global__ void k_mac_bc_z(T *u, T *v, T *w, BCDev bc, long long xs, long long ys, int nx, int ny, int nz) {
  pdl_entry();
  const int j = (int)(blockIdx.x * blockDim.x + threadIdx.x) - 1;
  const int i = (int)(blockIdx.y * blockDim.y + threadIdx.y) - 1;
  if (i > nx || j > ny) return;
  auto K = [&](int k) { return (long long)i * xs + (long long)j * ys + k; };
  if (bc.ty(FZ_NEG) == OCU_BC_PERIODIC) {
    w[K(-1)] = w[K(nz - 1)];
    u[K(-1)] = u[K(nz - 1)];
    v[K(-1)] = v[K(nz - 1)];
  } else if (bc.ty(FZ_NEG) == OCU_BC_FORCED_INFLOW_VARIABLE_SLIP) {
    const float f = 1.0f - 2.0f * bc.auxv(FZ_NEG);
    w[K(-1)] = (T)bc.val(FZ_NEG);
    w[K(0)] = (T)bc.val(FZ_NEG);
    u[K(-1)] = u[K(0)] * (T)f;
    v[K(-1)] = v[K(0)] * (T)f;
  }
  if (bc.ty(FZ_POS) == OCU_BC_PERIODIC) {
    w[K(nz)] = w[K(0)];
    w[K(nz + 1)] = w[K(1)];
    u[K(nz)] = u[K(0)];
    v[K(nz)] = v[K(0)];
  } else if (bc.ty(FZ_POS) == OCU_BC_FORCED_INFLOW_VARIABLE_SLIP) {
    const float f = 1.0f - 2.0f * bc.auxv(FZ_POS);
    w[K(nz)] = (T)bc.val(FZ_POS);
    w[K(nz + 1)] = (T)bc.val(FZ_POS);
    u[K(nz)] = u[K(nz - 1)] * (T)f;
    v[K(nz)] = v[K(nz - 1)] * (T)f;
  }
}

template <typename T>
ocu_status launch_mac_bc_level1(T *u, T *v, T *w, const ocu_layout &L, int nx, int ny, int nz,
                                const ocu_bc_set &bc, cudaStream_t s) {
  if (!bc_check_mac(bc))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] apply_3d_mac_boundary_conditions_level1 - invalid boundary condition types");
  if (L.gx < 1 || L.gy < 1 || L.gz < 1)
    return fail(OCU_ERR_LAYOUT, "[ERROR] apply_3d_mac_boundary_conditions_level1 - must have at least 1 ghost point");
  const BCDev d = to_dev(bc);
  dim3 b(32, 8);
  launch_pdl(k_mac_bc_x<T>, dim3((nz + 31) / 32, (ny + 7) / 8), b, 0, s, u, v, w, d, L.xstride, L.ystride, nx, ny, nz);
  OCU_TRY(check_launch("k_mac_bc_x"));
  launch_pdl(k_mac_bc_y<T>, dim3((nz + 31) / 32, (nx + 2 + 7) / 8), b, 0, s, u, v, w, d, L.xstride, L.ystride, nx, ny, nz);
  OCU_TRY(check_launch("k_mac_bc_y"));
  launch_pdl(k_mac_bc_z<T>, dim3((ny + 2 + 31) / 32, (nx + 2 + 7) / 8), b, 0, s, u, v, w, d, L.xstride, L.ystride, nx, ny, nz);
  return check_launch("k_mac_bc_z");
}

// ------------------------------------------------------------------------------------------
// clear / convert / linear combinations (grid3ddev.cu:25-85)
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_clear(T *buf, long long n, T value) {
  pdl_entry();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    buf[i] = value;
}

template <typename T, typename S>
__global__ void k_convert(T *dst, const S *src, long long n) {
  pdl_entry();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (T)src[i];
}

template <typename T>
__global__ void k_lincomb1(T *res, T a1, const T *g1, long long n) {
  pdl_entry();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    res[i] = g1[i] * a1;
}

template <typename T>
__global__ void k_lincomb2_1d(T *res, T a1, const T *g1, T a2, const T *g2, long long n) {
  pdl_entry();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    res[i] = g1[i] * a1 + g2[i] * a2;
}

template <typename T>
__global__ void k_lincomb2_3d(T *res, T a1, const T *g1, T a2, const T *g2, long long xs, long long ys,
                              int nx, int ny, int nz) {
  pdl_entry();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int i = blockIdx.z;
  if (k >= nz || j >= ny || i >= nx) return;
  const long long id = (long long)i * xs + (long long)j * ys + k;
  res[id] = g1[id] * a1 + g2[id] * a2;
}

// The same sum over 16-byte groups of a row: k = 0 of every row is 16-byte aligned (checked by
// the launcher), a row's last group may be partial.  Per element the arithmetic is unchanged.
template <typename T>
__global__ void k_lincomb2_3dv(T *res, T a1, const T *g1, T a2, const T *g2, long long xs, long long ys, int ny,
                               int nz, int cpr, long long nchunks) {
  pdl_entry();
  constexpr int V = 16 / (int)sizeof(T);
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < nchunks;
       c += (long long)gridDim.x * blockDim.x) {
    const long long row = c / cpr;
    const int k0 = (int)(c - row * cpr) * V;
    const int i = (int)(row / ny), j = (int)(row - (long long)i * ny);
    const long long id = (long long)i * xs + (long long)j * ys + k0;
    if (k0 + V <= nz) {
      if constexpr (sizeof(T) == 4) {
        const float4 x = *reinterpret_cast<const float4 *>(g1 + id), y = *reinterpret_cast<const float4 *>(g2 + id);
        float4 r;
        r.x = x.x * a1 + y.x * a2; r.y = x.y * a1 + y.y * a2;
        r.z = x.z * a1 + y.z * a2; r.w = x.w * a1 + y.w * a2;
        *reinterpret_cast<float4 *>(res + id) = r;
      } else {
        const double2 x = *reinterpret_cast<const double2 *>(g1 + id), y = *reinterpret_cast<const double2 *>(g2 + id);
        double2 r;
        r.x = x.x * a1 + y.x * a2; r.y = x.y * a1 + y.y * a2;
        *reinterpret_cast<double2 *>(res + id) = r;
      }
    } else {
      for (int e = 0; k0 + e < nz; e++) res[id + e] = g1[id + e] * a1 + g2[id + e] * a2;
    }
  }
}

static unsigned grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148LL * 32) b = 148LL * 32;
  if (b < 1) b = 1;
  return (unsigned)b;
}

template <typename T>
ocu_status launch_clear(T *buf, long long n, T value, cudaStream_t s) {
  launch_pdl(k_clear<T>, grid_for(n, 256), 256, 0, s, buf, n, value);
  return check_launch("k_clear");
}

template <typename T, typename S>
ocu_status launch_convert(T *dst, const S *src, long long n, cudaStream_t s) {
  launch_pdl(k_convert<T, S>, grid_for(n, 256), 256, 0, s, dst, src, n);
  return check_launch("k_convert");
}

template <typename T>
ocu_status launch_lincomb1(T *res, T a1, const T *g1, long long n, cudaStream_t s) {
  launch_pdl(k_lincomb1<T>, grid_for(n, 256), 256, 0, s, res, a1, g1, n);
  return check_launch("k_lincomb1");
}

// The reference switches to the interior-only kernel when more than 3% of the buffer is
// padding (grid3ddev.cu:312); otherwise it sweeps the whole buffer, ghosts included.
template <typename T>
ocu_status launch_lincomb2(T *res, const ocu_layout &L, T a1, const T *g1, T a2, const T *g2,
                           cudaStream_t s) {
  const long long waste = L.allocated - (long long)L.nx * L.ny * L.nz;
  if ((double)waste > 0.03 * (double)L.allocated) {
    const auto a16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    if (a16(res + L.shift) && a16(g1 + L.shift) && a16(g2 + L.shift) && (L.ystride * sizeof(T)) % 16 == 0 &&
        (L.xstride * sizeof(T)) % 16 == 0 && L.nx > 0 && L.ny > 0 && L.nz > 0) {
      constexpr int V = 16 / (int)sizeof(T);
      const int cpr = (L.nz + V - 1) / V;
      const long long nchunks = (long long)L.nx * L.ny * cpr;
      launch_pdl(k_lincomb2_3dv<T>, grid_for(nchunks, 256), 256, 0, s, res + L.shift, a1, g1 + L.shift, a2,
                 g2 + L.shift, L.xstride, L.ystride, L.ny, L.nz, cpr, nchunks);
      return check_launch("k_lincomb2_3dv");
    }
    dim3 grid((L.nz + 127) / 128, L.ny, L.nx);
    launch_pdl(k_lincomb2_3d<T>, grid, 128, 0, s, res + L.shift, a1, g1 + L.shift, a2, g2 + L.shift, L.xstride,
               L.ystride, L.nx, L.ny, L.nz);
    return check_launch("k_lincomb2_3d");
  }
  launch_pdl(k_lincomb2_1d<T>, grid_for(L.allocated, 256), 256, 0, s, res, a1, g1, a2, g2, L.allocated);
  return check_launch("k_lincomb2_1d");
}

// ------------------------------------------------------------------------------------------
// Reductions in the reference fold order (grid3dops.cu:26-130, grid1dops.cu:33-115), one
// launch: block b folds rows [256b, 256b+256) -- row value = lane-strided fold over k then a
// 16/8/4/2/1 shuffle tree -- then a 256-wide stride-halving tree; the last block to finish
// folds the block partials with further 256-wide trees.  Deterministic.
// ------------------------------------------------------------------------------------------
template <typename T>
struct RedOp {
  int op;
  __device__ __forceinline__ T identity() const {
    if (op == OCU_REDUCE_MAX) return sizeof(T) == 4 ? (T)-3.40282347e+38f : (T)-1e100;
    if (op == OCU_REDUCE_MIN) return sizeof(T) == 4 ? (T)3.40282347e+38f : (T)1e100;
    return (T)0;
  }
  __device__ __forceinline__ T process(T a) const {
    if (op == OCU_REDUCE_MAXABS) return fabs(a);
    if (op == OCU_REDUCE_SQRSUM) return a * a;
    return a;
  }
  __device__ __forceinline__ T reduce(T a, T b) const {
    switch (op) {
      case OCU_REDUCE_MAXABS:
      case OCU_REDUCE_MAX: return fmax(a, b);
      case OCU_REDUCE_MIN: return fmin(a, b);
      case OCU_REDUCE_CHECKNAN: return isfinite((float)a) ? b : a;
      default: return a + b;
    }
  }
};

template <typename T>
__device__ __forceinline__ void block_tree_256(T *sh, const RedOp<T> &op) {
  for (int stride = 128; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride) sh[threadIdx.x] = op.reduce(sh[threadIdx.x], sh[threadIdx.x + stride]);
    __syncthreads();
  }
}

constexpr int kReduceThreads = 512;  // 16 warps, 16 of a block's 256 rows each; two blocks per SM

template <typename T>
__global__ void __launch_bounds__(kReduceThreads, 2) k_reduce(const T *origin, long long xs, long long ys, int nx, int ny, int nz,
                                                RedOp<T> op, T *partial, unsigned *counter, double *result) {
  pdl_entry();
  __shared__ T sh[256];
  __shared__ bool last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long nrows = (long long)nx * ny;
  const long long row0 = (long long)blockIdx.x * 256;
  // A warp folds its RB rows together: each row in its own order (lane-strided over k, then
  // the shuffle tree), the loads of the RB rows interleaved so that they are in flight
  // together.  Rows beyond nrows carry the identity, as in reduce_per_cta.
  constexpr int RW = 256 / (kReduceThreads / 32);  // rows of a warp
  constexpr int RB = 8;
  static_assert(RW % RB == 0, "rows of a warp in whole groups");
  for (int r0 = 0; r0 < RW; r0 += RB) {
    T acc[RB];
    const T *base[RB];
    bool ok[RB];
    // consecutive rows: one division for the first, then step j (wrapping into i)
    const long long qb = row0 + warp * RW + r0;
    int i = (int)(qb / ny), j = (int)(qb - (long long)i * ny);
#pragma unroll
    for (int r = 0; r < RB; r++) {
      ok[r] = qb + r < nrows;
      acc[r] = op.identity();
      base[r] = ok[r] ? origin + (long long)i * xs + (long long)j * ys : origin;
      if (++j == ny) {
        j = 0;
        ++i;
      }
    }
    // per step of k the loads of all RB rows first (a row beyond nrows reads row 0, which
    // exists, and is ignored), then the folds, each row in its own order
    for (int k = lane; k < nz; k += 32) {
      T v[RB];
#pragma unroll
      for (int r = 0; r < RB; r++) v[r] = base[r][k];
#pragma unroll
      for (int r = 0; r < RB; r++)
        if (ok[r]) acc[r] = k == lane ? op.process(v[r]) : op.reduce(op.process(v[r]), acc[r]);
    }
#pragma unroll
    for (int r = 0; r < RB; r++) {
      T a = acc[r];
      for (int o = 16; o > 0; o >>= 1) {
        T other = __shfl_down_sync(0xffffffffu, a, o);
        a = op.reduce(a, other);
      }
      if (lane == 0) sh[warp * RW + r0 + r] = a;
    }
  }
  __syncthreads();
  block_tree_256(sh, op);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = sh[0];
    __threadfence();
    const unsigned ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // fold partials: passes of 256-wide trees until one value remains (grid1dops.cu:95-106)
  long long count = gridDim.x;
  volatile T *vp = partial;
  while (count > 1) {
    const long long nb = (count + 255) / 256;
    for (long long b = 0; b < nb; b++) {
      const long long idx = b * 256 + threadIdx.x;
      if (threadIdx.x < 256) sh[threadIdx.x] = idx < count ? vp[idx] : op.identity();
      __syncthreads();
      block_tree_256(sh, op);
      if (threadIdx.x == 0) vp[b] = sh[0];
      __syncthreads();
    }
    count = nb;
  }
  if (threadIdx.x == 0) {
    *result = (double)vp[0];
    *counter = 0;  // ready for the next launch on this scratch
  }
}

size_t reduce_scratch_bytes(const ocu_layout &L, size_t elem) {
  const long long nrows = (long long)L.nx * L.ny;
  const long long blocks = (nrows + 255) / 256;
  return (size_t)(blocks > 0 ? blocks : 1) * elem + 64;
}

template <typename T>
ocu_status launch_reduce(const T *origin, const ocu_layout &L, int op, void *d_scratch,
                         double *d_result, cudaStream_t s) {
  const long long nrows = (long long)L.nx * L.ny;
  const long long blocks = (nrows + 255) / 256;
  if (blocks < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] reduce_with_operator - empty grid");
  // the ticket counter sits at a fixed offset so scratch can be shared by reductions of
  // different sizes on one stream; the block partials follow it
  unsigned *counter = reinterpret_cast<unsigned *>(d_scratch);
  T *partial = reinterpret_cast<T *>(reinterpret_cast<char *>(d_scratch) + 64);
  RedOp<T> r{op};
  launch_pdl(k_reduce<T>, (unsigned)blocks, kReduceThreads, 0, s, origin, L.xstride, L.ystride, L.nx, L.ny, L.nz, r, partial,
             counter, d_result);
  return check_launch("k_reduce");
}

#define INST(T)                                                                                               \
  template ocu_status launch_bc_level1<T>(T *, const ocu_layout &, const ocu_bc_set &, double, double, double, \
                                          cudaStream_t);                                                      \
  template ocu_status launch_bc_nocorners_dev<T>(T *, const ocu_layout &, const ocu_bc_set &, double, double,  \
                                                 double, cudaStream_t);                                       \
  template ocu_status launch_mac_bc_level1<T>(T *, T *, T *, const ocu_layout &, int, int, int,                \
                                              const ocu_bc_set &, cudaStream_t);                              \
  template ocu_status launch_clear<T>(T *, long long, T, cudaStream_t);                                        \
  template ocu_status launch_lincomb1<T>(T *, T, const T *, long long, cudaStream_t);                          \
  template ocu_status launch_lincomb2<T>(T *, const ocu_layout &, T, const T *, T, const T *, cudaStream_t);   \
  template ocu_status launch_reduce<T>(const T *, const ocu_layout &, int, void *, double *, cudaStream_t);
INST(float)
INST(double)
#undef INST
template ocu_status launch_convert<float, double>(float *, const double *, long long, cudaStream_t);
template ocu_status launch_convert<double, float>(double *, const float *, long long, cudaStream_t);
template ocu_status launch_convert<float, float>(float *, const float *, long long, cudaStream_t);
template ocu_status launch_convert<double, double>(double *, const double *, long long, cudaStream_t);

}  // namespace ocub
