// Grid kernels: ghost fills, clear/convert/axpy and deterministic reductions.
//
// All arithmetic reproduces the reference expression order; the library is compiled with
// --fmad=false so every product and sum is rounded exactly as written.
#include <algorithm>
#include <cfloat>
#include <cstdint>

#include <type_traits>

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
__global__ void k_lincomb2_1d(T *res, T a1, const T *g1, Coef<T> a2c, const T *g2, long long n) {
  pdl_entry();
  const T a2 = a2c.get();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    res[i] = g1[i] * a1 + g2[i] * a2;
}

template <typename T>
__global__ void k_lincomb2_3d(T *res, T a1, const T *g1, Coef<T> a2c, const T *g2, long long xs, long long ys,
                              int nx, int ny, int nz) {
  pdl_entry();
  const T a2 = a2c.get();
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
__global__ void k_lincomb2_3dv(T *res, T a1, const T *g1, Coef<T> a2c, const T *g2, long long xs, long long ys,
                               int ny, int nz, int cpr, long long nchunks) {
  pdl_entry();
  const T a2 = a2c.get();
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

// The velocity update of a time step over u, v and w (one layout) in one pass: x = x * 1 + d * a2,
// then, with Adams-Bashforth history, x = x * 1 + l * a3 -- the reference's one or two
// linear_combination calls per component, each rounded as there (grid3ddev.cu:283-349).
template <typename T>
struct UpdateSet {
  T *x[3];
  const T *d[3], *l[3];
};

template <typename T, bool AB2>
__global__ void k_update3_3dv(const __grid_constant__ UpdateSet<T> S, Coef<T> a2c, Coef<T> a3c, long long xs,
                              long long ys, int ny, int nz, int cpr, long long nchunks) {
  pdl_entry();
  const T a2 = a2c.get(), a3 = a3c.get();
  constexpr int V = 16 / (int)sizeof(T);
  using Vec = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < 3 * nchunks;
       c += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(c / nchunks);
    const long long cc = c - f * nchunks;
    T *x = f == 0 ? S.x[0] : (f == 1 ? S.x[1] : S.x[2]);
    const T *d = f == 0 ? S.d[0] : (f == 1 ? S.d[1] : S.d[2]);
    const T *l = f == 0 ? S.l[0] : (f == 1 ? S.l[1] : S.l[2]);
    const long long row = cc / cpr;
    const int k0 = (int)(cc - row * cpr) * V;
    const int i = (int)(row / ny), j = (int)(row - (long long)i * ny);
    const long long id = (long long)i * xs + (long long)j * ys + k0;
    if (k0 + V <= nz) {
      Vec xv = *reinterpret_cast<const Vec *>(x + id);
      const Vec dv = *reinterpret_cast<const Vec *>(d + id);
      T *xe = reinterpret_cast<T *>(&xv);
      const T *de = reinterpret_cast<const T *>(&dv);
#pragma unroll
      for (int e = 0; e < V; e++) xe[e] = xe[e] * (T)1 + de[e] * a2;
      if (AB2) {
        const Vec lv = *reinterpret_cast<const Vec *>(l + id);
        const T *le = reinterpret_cast<const T *>(&lv);
#pragma unroll
        for (int e = 0; e < V; e++) xe[e] = xe[e] * (T)1 + le[e] * a3;
      }
      *reinterpret_cast<Vec *>(x + id) = xv;
    } else {
      for (int e = 0; k0 + e < nz; e++) {
        T v = x[id + e] * (T)1 + d[id + e] * a2;
        if (AB2) v = v * (T)1 + l[id + e] * a3;
        x[id + e] = v;
      }
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

// OCU_ERR_UNSUPPORTED when the interior-only 16-byte form would not be the one the separate
// linear combinations take (the caller then launches those).
template <typename T>
ocu_status launch_update3(T *const *x, const T *const *d, const T *const *l, const ocu_layout &L, Coef<T> a2,
                          Coef<T> a3, cudaStream_t s) {
  const long long waste = L.allocated - (long long)L.nx * L.ny * L.nz;
  const auto a16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  bool ok = (double)waste > 0.03 * (double)L.allocated && (L.ystride * sizeof(T)) % 16 == 0 &&
            (L.xstride * sizeof(T)) % 16 == 0 && L.nx > 0 && L.ny > 0 && L.nz > 0;
  for (int f = 0; f < 3 && ok; f++)
    ok = a16(x[f] + L.shift) && a16(d[f] + L.shift) && (!l || a16(l[f] + L.shift));
  if (!ok) return OCU_ERR_UNSUPPORTED;
  constexpr int V = 16 / (int)sizeof(T);
  const int cpr = (L.nz + V - 1) / V;
  const long long nchunks = (long long)L.nx * L.ny * cpr;
  UpdateSet<T> S;
  for (int f = 0; f < 3; f++) {
    S.x[f] = x[f] + L.shift;
    S.d[f] = d[f] + L.shift;
    S.l[f] = l ? l[f] + L.shift : nullptr;
  }
  if (l)
    launch_pdl(k_update3_3dv<T, true>, grid_for(3 * nchunks, 256), 256, 0, s, S, a2, a3, (long long)L.xstride,
               (long long)L.ystride, L.ny, L.nz, cpr, nchunks);
  else
    launch_pdl(k_update3_3dv<T, false>, grid_for(3 * nchunks, 256), 256, 0, s, S, a2, a3, (long long)L.xstride,
               (long long)L.ystride, L.ny, L.nz, cpr, nchunks);
  return check_launch("k_update3_3dv");
}

// The reference switches to the interior-only kernel when more than 3% of the buffer is
// padding (grid3ddev.cu:312); otherwise it sweeps the whole buffer, ghosts included.
template <typename T>
ocu_status launch_lincomb2(T *res, const ocu_layout &L, T a1, const T *g1, Coef<T> a2, const T *g2,
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

// DOT: the folded value of cell k is origin[k] * origin2[k] rounded to T (a pointwise product
// grid reduced with the sum, without storing the product grid).
template <typename T, bool DOT = false>
__global__ void __launch_bounds__(kReduceThreads, 2) k_reduce(const T *origin, const T *origin2, long long xs, long long ys,
                                                              int nx, int ny, int nz, RedOp<T> op, T *partial,
                                                              unsigned *counter, double *result) {
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
  constexpr int RB = (DOT && sizeof(T) == 8) ? 4 : 8;  // rows in flight; each row keeps its own fold
  static_assert(RW % RB == 0, "rows of a warp in whole groups");
  for (int r0 = 0; r0 < RW; r0 += RB) {
    T acc[RB];
    const T *base[RB];
    const T *base2[RB];
    bool ok[RB];
    // consecutive rows: one division for the first, then step j (wrapping into i)
    const long long qb = row0 + warp * RW + r0;
    int i = (int)(qb / ny), j = (int)(qb - (long long)i * ny);
#pragma unroll
    for (int r = 0; r < RB; r++) {
      ok[r] = qb + r < nrows;
      acc[r] = op.identity();
      base[r] = ok[r] ? origin + (long long)i * xs + (long long)j * ys : origin;
      base2[r] = DOT ? (ok[r] ? origin2 + (long long)i * xs + (long long)j * ys : origin2) : nullptr;
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
      for (int r = 0; r < RB; r++) v[r] = DOT ? base[r][k] * base2[r][k] : base[r][k];
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

// Max, min and max-abs in one pass: exact in any fold order, so no partials are kept.  Each warp
// folds one group of rows (read with 16-byte loads along k, a ragged row end with scalar loads,
// all the group's loads in flight together), the block folds its warps, and the block's value
// enters an unsigned key in the scratch header with atomicMax (an order-preserving encoding of
// the float; min as its complement); the last block decodes it and clears the key and the
// ticket for the next launch.  Folds start from NaN (fmax / fmin drop a NaN operand), so the
// result is the extremum of the grid's non-NaN values -- what the reference-order fold gives
// whenever the grid holds one -- and NaN when it holds none.
template <typename T>
__device__ __forceinline__ T red_nan();
template <>
__device__ __forceinline__ float red_nan<float>() { return __int_as_float(0x7fffffff); }
template <>
__device__ __forceinline__ double red_nan<double>() { return __longlong_as_double(0x7fffffffffffffffLL); }

template <typename T>
struct MMKey;
template <>
struct MMKey<float> {
  using K = unsigned;
  __device__ static K enc(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  }
  __device__ static float dec(K k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k); }
};
template <>
struct MMKey<double> {
  using K = unsigned long long;
  __device__ static K enc(double f) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(f);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
  }
  __device__ static double dec(K k) {
    return __longlong_as_double((long long)((k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k));
  }
};

// the operation fixed at compile time (a run-time switch in the unrolled loads spilled)
template <typename T, int OP>
struct MinMaxOp {
  __device__ __forceinline__ T process(T a) const { return OP == OCU_REDUCE_MAXABS ? fabs(a) : a; }
  __device__ __forceinline__ T reduce(T a, T b) const { return OP == OCU_REDUCE_MIN ? fmin(a, b) : fmax(a, b); }
};

constexpr int kMMThreads = 256;

template <typename T, bool VEC>
constexpr int mm_rows() { return (VEC && sizeof(T) == 4) ? 6 : 4; }  // rows of a warp (no spills)

// Up to three grids in one launch (the CFL step reduces u, v and w): blocks [b0[g], b0[g+1])
// fold grid g into key g; one ticket for the launch.
template <typename T>
struct MMGrids {
  const T *o0, *o1, *o2;
  long long xs, ys;       // shared strides
  int nx0, nx1, nx2, ny0, ny1, ny2, nz0, nz1, nz2;
  unsigned b1, b2;        // first blocks of grids 1 and 2
  int n;                  // grids
};

template <typename T, bool VEC, int OP>
__global__ void __launch_bounds__(kMMThreads, 4) k_reduce_mm(const __grid_constant__ MMGrids<T> G, unsigned *counter,
                                                          typename MMKey<T>::K *keys, double *results) {
  pdl_entry();
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  using K = typename MMKey<T>::K;
  constexpr int W = sizeof(V) / sizeof(T);
  constexpr int NW = kMMThreads / 32, RB = mm_rows<T, VEC>();
  const MinMaxOp<T, OP> op;
  __shared__ T sh[NW];
  __shared__ bool last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this block's grid (selects: an indexed parameter array would go to local memory)
  const int g = blockIdx.x >= G.b2 ? 2 : (blockIdx.x >= G.b1 ? 1 : 0);
  const T *origin = g == 2 ? G.o2 : (g == 1 ? G.o1 : G.o0);
  const int ny = g == 2 ? G.ny2 : (g == 1 ? G.ny1 : G.ny0);
  const int nz = g == 2 ? G.nz2 : (g == 1 ? G.nz1 : G.nz0);
  const int nx = g == 2 ? G.nx2 : (g == 1 ? G.nx1 : G.nx0);
  const unsigned blk = blockIdx.x - (g == 2 ? G.b2 : (g == 1 ? G.b1 : 0u));
  const unsigned nblk = (g == 2 ? gridDim.x : (g == 1 ? G.b2 : G.b1)) - (g == 2 ? G.b2 : (g == 1 ? G.b1 : 0u));
  const long long xs = G.xs, ys = G.ys;
  const long long nrows = (long long)nx * ny;
  T acc = red_nan<T>();
  // the grid's blocks take the groups of RB consecutive rows in turn (one resident wave: the
  // atomic and the ticket at a block's end are paid once per block)
  for (long long grp = (long long)blk * NW + warp; grp * RB < nrows; grp += (long long)nblk * NW) {
  const T *base[RB];
  bool ok[RB];
  // consecutive rows: one division for the first, then step j (wrapping into i)
  const long long qb = grp * RB;
  int i = (int)(qb / ny), j = (int)(qb - (long long)i * ny);
#pragma unroll
  for (int r = 0; r < RB; r++) {
    ok[r] = qb + r < nrows;
    base[r] = ok[r] ? origin + (long long)i * xs + (long long)j * ys : origin;
    if (++j == ny) {
      j = 0;
      ++i;
    }
  }
  if (VEC) {
    const int nzv = nz - nz % W;  // whole vectors; the ragged end of each row below
    for (int k = nzv + lane; k < nz; k += 32)
#pragma unroll
      for (int r = 0; r < RB; r++)
        if (ok[r]) acc = op.reduce(acc, op.process(base[r][k]));
    for (int k = lane * W; k < nzv; k += 32 * W) {
      V v[RB];
#pragma unroll
      for (int r = 0; r < RB; r++)
        if (ok[r]) v[r] = *reinterpret_cast<const V *>(base[r] + k);
#pragma unroll
      for (int r = 0; r < RB; r++)
        if (ok[r]) {
          const T *e = reinterpret_cast<const T *>(&v[r]);
#pragma unroll
          for (int c = 0; c < W; c++) acc = op.reduce(acc, op.process(e[c]));
        }
    }
  } else {
    for (int k = lane; k < nz; k += 32) {
      T v[RB];
#pragma unroll
      for (int r = 0; r < RB; r++)
        if (ok[r]) v[r] = base[r][k];
#pragma unroll
      for (int r = 0; r < RB; r++)
        if (ok[r]) acc = op.reduce(acc, op.process(v[r]));
    }
  }
  }
  for (int o = 16; o > 0; o >>= 1) acc = op.reduce(acc, __shfl_down_sync(0xffffffffu, acc, o));
  if (lane == 0) sh[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    T a = sh[0];
    for (int w = 1; w < NW; w++) a = op.reduce(a, sh[w]);
    if (a == a) {  // a block of NaNs only contributes nothing
      const K kv = MMKey<T>::enc(a);
      atomicMax(keys + g, OP == OCU_REDUCE_MIN ? ~kv : kv);
    }
    __threadfence();
    const unsigned ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x >= G.n) return;
  __threadfence();
  const K kv = atomicMax(keys + threadIdx.x, (K)0);  // the final key (max with the empty key leaves it)
  results[threadIdx.x] = kv == 0 ? (double)red_nan<T>() : (double)MMKey<T>::dec(OP == OCU_REDUCE_MIN ? ~kv : kv);
  keys[threadIdx.x] = 0;
  if (threadIdx.x == 0) *counter = 0;
}

// n (1..3) grids sharing strides: min, max or max-abs of each into results[0..n); scratch: the
// ticket at +0, the n keys from +8 (inside the 64-byte header every reduction scratch has), all
// zero between launches.
template <typename T>
ocu_status launch_minmax(const T *const *origins, const ocu_layout *const *lays, int n, int op, void *d_scratch,
                         double *d_results, cudaStream_t s) {
  using K = typename MMKey<T>::K;
  static_assert(sizeof(K) <= 8, "key slots are 8 bytes");
  if (n < 1 || n > 3) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] reduce - %d grids", n);
  constexpr int W = 16 / sizeof(T);
  bool vec = true;
  MMGrids<T> G{};
  G.n = n;
  G.xs = lays[0]->xstride;
  G.ys = lays[0]->ystride;
  unsigned start[3] = {0, 0, 0}, total = 0;
  for (int g = 0; g < n; g++) {
    if (lays[g]->xstride != G.xs || lays[g]->ystride != G.ys)
      return fail(OCU_ERR_LAYOUT, "[ERROR] reduce - grids of one launch must share strides");
    vec = vec && G.xs % W == 0 && G.ys % W == 0 && reinterpret_cast<uintptr_t>(origins[g]) % 16 == 0;
  }
  // one resident wave, shared among the grids in proportion to their rows (at least one block,
  // at most one per block's worth of rows each)
  static int wave = 0;
  if (!wave) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_reduce_mm<T, true, OCU_REDUCE_MAXABS>, kMMThreads, 0);
    wave = sms > 0 && per > 0 ? sms * per : 148 * 8;
  }
  const long long rpb = (long long)(kMMThreads / 32) * (vec ? mm_rows<T, true>() : mm_rows<T, false>());
  long long rows[3] = {0, 0, 0}, all = 0;
  for (int g = 0; g < n; g++) {
    rows[g] = (long long)lays[g]->nx * lays[g]->ny;
    if (rows[g] < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] reduce_with_operator - empty grid");
    all += rows[g];
  }
  for (int g = 0; g < n; g++) {
    long long b = (long long)((double)wave * rows[g] / all);
    b = std::max(1LL, std::min(b, (rows[g] + rpb - 1) / rpb));
    start[g] = total;
    total += (unsigned)b;
  }
  G.o0 = origins[0]; G.o1 = n > 1 ? origins[1] : origins[0]; G.o2 = n > 2 ? origins[2] : origins[0];
  G.nx0 = lays[0]->nx; G.ny0 = lays[0]->ny; G.nz0 = lays[0]->nz;
  G.nx1 = lays[n > 1 ? 1 : 0]->nx; G.ny1 = lays[n > 1 ? 1 : 0]->ny; G.nz1 = lays[n > 1 ? 1 : 0]->nz;
  G.nx2 = lays[n > 2 ? 2 : 0]->nx; G.ny2 = lays[n > 2 ? 2 : 0]->ny; G.nz2 = lays[n > 2 ? 2 : 0]->nz;
  G.b1 = n > 1 ? start[1] : total;
  G.b2 = n > 2 ? start[2] : total;
  unsigned *counter = reinterpret_cast<unsigned *>(d_scratch);
  K *keys = reinterpret_cast<K *>(reinterpret_cast<char *>(d_scratch) + 8);
#define OCU_MM_LAUNCH(V, O) \
  launch_pdl(k_reduce_mm<T, V, O>, total, kMMThreads, 0, s, G, counter, keys, d_results)
  if (vec) {
    if (op == OCU_REDUCE_MAXABS) OCU_MM_LAUNCH(true, OCU_REDUCE_MAXABS);
    else if (op == OCU_REDUCE_MAX) OCU_MM_LAUNCH(true, OCU_REDUCE_MAX);
    else OCU_MM_LAUNCH(true, OCU_REDUCE_MIN);
  } else {
    if (op == OCU_REDUCE_MAXABS) OCU_MM_LAUNCH(false, OCU_REDUCE_MAXABS);
    else if (op == OCU_REDUCE_MAX) OCU_MM_LAUNCH(false, OCU_REDUCE_MAX);
    else OCU_MM_LAUNCH(false, OCU_REDUCE_MIN);
  }
#undef OCU_MM_LAUNCH
  return check_launch("k_reduce_mm");
}

// A few doubles from device memory into pinned host memory by a one-warp kernel.  Pinned host
// memory is mapped into the device's address space under unified addressing, so the stores
// cross PCIe as the kernel's own writes: a host-blocking readback of a norm is not queued on
// the device-to-host copy engine behind a large transfer that another stream has issued.
__global__ void k_readback(const double *__restrict__ src, double *dst, int n) {
  pdl_entry();
  const int i = threadIdx.x;
  if (i < n) dst[i] = src[i];
  __threadfence_system();
}

ocu_status launch_readback(const double *src, double *host_pinned, int n, cudaStream_t s) {
  if (n < 1 || n > 32) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] readback - bad count %d", n);
  launch_pdl(k_readback, dim3(1), dim3(32), 0, s, src, host_pinned, n);
  return check_launch("k_readback");
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
  if (op == OCU_REDUCE_MAX || op == OCU_REDUCE_MIN || op == OCU_REDUCE_MAXABS) {
    const T *o[1] = {origin};
    const ocu_layout *l[1] = {&L};
    return launch_minmax<T>(o, l, 1, op, d_scratch, d_result, s);
  }
  launch_pdl(k_reduce<T, false>, (unsigned)blocks, kReduceThreads, 0, s, origin, (const T *)nullptr, L.xstride,
             L.ystride, L.nx, L.ny, L.nz, r, partial, counter, d_result);
  return check_launch("k_reduce");
}

// sum over the interior of a * b (both in layout L), in the reference fold order of
// reduce_sum over the product grid (sol_pcgpressure3d.cu:257-287)
template <typename T>
ocu_status launch_dot(const T *a, const T *b, const ocu_layout &L, void *d_scratch, double *d_result, cudaStream_t s) {
  const long long nrows = (long long)L.nx * L.ny;
  const long long blocks = (nrows + 255) / 256;
  if (blocks < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] dot product - empty grid");
  unsigned *counter = reinterpret_cast<unsigned *>(d_scratch);
  T *partial = reinterpret_cast<T *>(reinterpret_cast<char *>(d_scratch) + 64);
  RedOp<T> r{OCU_REDUCE_SUM};
  launch_pdl(k_reduce<T, true>, (unsigned)blocks, kReduceThreads, 0, s, a, b, L.xstride, L.ystride, L.nx, L.ny, L.nz,
             r, partial, counter, d_result);
  return check_launch("k_reduce_dot");
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
  template ocu_status launch_lincomb2<T>(T *, const ocu_layout &, T, const T *, Coef<T>, const T *, cudaStream_t); \
  template ocu_status launch_reduce<T>(const T *, const ocu_layout &, int, void *, double *, cudaStream_t);    \
  template ocu_status launch_update3<T>(T *const *, const T *const *, const T *const *, const ocu_layout &, Coef<T>, \
                                        Coef<T>, \
                                        cudaStream_t);                                                        \
  template ocu_status launch_dot<T>(const T *, const T *, const ocu_layout &, void *, double *, cudaStream_t);  \
  template ocu_status launch_minmax<T>(const T *const *, const ocu_layout *const *, int, int, void *, double *,  \
                                       cudaStream_t);
INST(float)
INST(double)
#undef INST
template ocu_status launch_convert<float, double>(float *, const double *, long long, cudaStream_t);
template ocu_status launch_convert<double, float>(double *, const float *, long long, cudaStream_t);
template ocu_status launch_convert<float, float>(float *, const float *, long long, cudaStream_t);
template ocu_status launch_convert<double, double>(double *, const double *, long long, cudaStream_t);

}  // namespace ocub
