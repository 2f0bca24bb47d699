// Fused multigrid kernels (same arithmetic as kernels_mg.cu, fewer launches and bytes):
//   - colour sweep and prolongation that also write the ghosts of the cells they update;
//   - residual + 8-cell restriction + norm partials in one pass (r is never written);
//   - residual + norms (+ optional FP32 down-cast) for the level-0 checks and the refinement
//     solver;
//   - a single-CTA kernel that runs the coarse end of a V-cycle (all levels at or below a few
//     thousand cells) with __syncthreads between phases instead of one launch per operation,
//     staged in shared memory when the levels fit (about 200 KB).
// Norm partials follow the reference fold order exactly (grid3dops.cu:26-130): for each fine
// (i,j) row, lane t folds k = t, t+32, ... and the 32 lanes fold 16/8/4/2/1; rows are folded by
// 256-wide trees (grid1dops.cu:33-115) in k_fold_rows.
#include <atomic>
#include <cstring>

#include "bc_device.cuh"
#include "ghost_emit.cuh"
#include "mg_fused.h"
#include "ocu_internal.h"
#include "relax_math.cuh"

namespace ocub {

// One colour update of cell (i,j,k).  In a block that holds no cell of the outer layer the
// diagonal is c.ld exactly (every face term is skipped) and there are no ghost writes.  I is the
// index type: int when the whole allocation fits in 2^31 elements.
// ZFAST: rows off the x and y faces in an edge block (an edge block only through z) take a short
// path -- relax_dg's sequence reduces to the z terms (the FP64 table holds ld there) and the
// cell's only ghosts are its z ghosts.  Used where it measured faster: the large FP64 levels and
// the ensemble sweeps (on the small levels the longer kernel was slower).
template <typename T, typename I, bool ZFAST = false>
__device__ __forceinline__ void color_cell(T *__restrict__ u, const T *__restrict__ b, I xs, I ys, int i, int j,
                                           int k, int nx, int ny, int nz, const RelaxCoefD<T> &c,
                                           const T *__restrict__ diag, bool edge_block, const GhostEmit<T> &ge) {
  const I id = (I)i * xs + (I)j * ys + k;
  if (!edge_block) {
    const T uc = u[id];
    const T res = relax_res<T>(uc, b[id], u[id - 1], u[id + 1], u[id - ys], u[id + ys], u[id - xs], u[id + xs], c);
    u[id] = uc + c.omega * res / c.ld;
    return;
  }
  if (ZFAST && i > 0 && i < nx - 1 && j > 0 && j < ny - 1) {
    const T uc = u[id];
    const T res = relax_res<T>(uc, b[id], u[id - 1], u[id + 1], u[id - ys], u[id + ys], u[id - xs], u[id + xs], c);
    T dg = c.ld;
    if (k == nz - 1) dg += c.zp;
    if (k == 0) dg += c.zn;
    const T nv = uc + c.omega * res / dg;
    u[id] = nv;
    const int tn = ge.bc.type[FZ_NEG], tp = ge.bc.type[FZ_POS];
    if (k == 0) {
      if (tn == OCU_BC_DIRICHELET || tn == OCU_BC_NEUMANN) u[id - 1] = ge.template rule<FZ_NEG>(nv, ge.hz);
      if (tp == OCU_BC_PERIODIC) u[id + nz] = ge.template rule<FZ_POS>(nv, ge.hz);
    }
    if (k == nz - 1) {
      if (tp == OCU_BC_DIRICHELET || tp == OCU_BC_NEUMANN) u[id + 1] = ge.template rule<FZ_POS>(nv, ge.hz);
      if (tn == OCU_BC_PERIODIC) u[id - nz] = ge.template rule<FZ_NEG>(nv, ge.hz);
    }
    return;
  }
  const T nv = relax_value<T>(u[id], b[id], u[id - 1], u[id + 1], u[id - ys], u[id + ys], u[id - xs], u[id + xs], i,
                              j, k, nx, ny, nz, c, diag);
  u[id] = nv;
  ge.emit(i, j, k, nv);
}

__device__ __forceinline__ bool color_edge_block(int bx, int by, int bz, int nx, int ny, int nz) {
  return bx == 0 || (bx + 1) * (int)blockDim.x * 2 >= nz || by == 0 || (by + 1) * (int)blockDim.y >= ny || bz == 0 ||
         (bz + 1) * (int)blockDim.z >= nx;
}

// Colour sweep + ghost writes: thread (t, j, i), k = 2t + parity.
template <typename T, typename I, bool ZFAST>
__global__ void __launch_bounds__(256, 6) k_relax_color_emit(T *__restrict__ u, const T *__restrict__ b,
                                                                         I xs, I ys,
                                                          int nx, int ny, int nz, int color, RelaxCoefD<T> c,
                                                          const T *__restrict__ diag,
                                                          const __grid_constant__ GhostEmit<T> ge) {
  pdl_entry();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  // block row 0 takes the last plane block: the blocks of both face planes (all edge blocks,
  // the slowest) run first
  const int bz = blockIdx.z == 0 ? gridDim.z - 1 : blockIdx.z - 1;
  const int i = bz * blockDim.z + threadIdx.z;
  const bool edge_block = color_edge_block(blockIdx.x, blockIdx.y, bz, nx, ny, nz);
  if (i >= nx || j >= ny || t >= nz / 2) return;
  color_cell<T, I, ZFAST>(u, b, xs, ys, i, j, 2 * t + ((i + j + color) & 1), nx, ny, nz, c, diag, edge_block, ge);
}

// FP32 colour sweep with 128-bit accesses: a thread owns four consecutive cells of a row (two of
// each colour) and updates its two cells of the sweep's colour.  Its row neighbours come from
// the same float4 or, across the float4 boundary, from the adjacent lanes; u of the rows j +- 1
// and planes i +- 1 and b are float4 loads (ghost rows and planes included); the two new values
// go back with one float4 store (the other two entries rewritten unchanged: nothing else writes
// them in this launch).  A warp covers 128 consecutive cells of one row (nz a multiple of 128).
// The diagonal adds the face terms of relax_dg in its order (x, y only on face rows).  Rows on a
// j or i face write every ghost of their cells (GhostEmit); in the other rows only the z-face
// ghosts exist, and they are stored directly with the z rule (for a cell whose i and j are
// interior, GhostEmit writes exactly that one ghost).  The planes i = 0 and nx - 1 hold the
// slowest rows, so their blocks are scheduled first.
template <typename T>
__device__ __forceinline__ T v4_update(T uc, T bv, T zm, T zp, T ym, T yp, T xm, T xp, int i, int j, int k, int nx,
                                       int ny, int nz, bool face_row, const RelaxCoefD<T> &c) {
  const T res = relax_res<T>(uc, bv, zm, zp, ym, yp, xm, xp, c);
  T dg = c.ld;
  if (face_row) {
    if (i == nx - 1) dg += c.xp;
    if (i == 0) dg += c.xn;
    if (j == ny - 1) dg += c.yp;
    if (j == 0) dg += c.yn;
  }
  if (k == nz - 1) dg += c.zp;
  if (k == 0) dg += c.zn;
  return uc + c.omega * res / dg;
}

__global__ void __launch_bounds__(256, 6) k_relax_color_v4(float *__restrict__ u, const float *__restrict__ b, int xs,
                                                        int ys, int nx, int ny, int nz, int color,
                                                        RelaxCoefD<float> c, const __grid_constant__ GhostEmit<float> ge) {
  pdl_entry();
  const int lane = threadIdx.x;
  const int k4 = (blockIdx.x * 32 + lane) * 4;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  // block row 0 takes the last plane pair, the others shift by one: both face planes run first
  const int bz = blockIdx.z == 0 ? gridDim.z - 1 : blockIdx.z - 1;
  const int i = bz * blockDim.z + threadIdx.z;
  if (i >= nx || j >= ny) return;  // whole warps (one row each)
  const int par = (i + j + color) & 1;
  const bool face_row = i == 0 || i == nx - 1 || j == 0 || j == ny - 1;
  const int base = i * xs + j * ys + k4;
  const float4 U = *reinterpret_cast<const float4 *>(u + base);
  const float4 B = *reinterpret_cast<const float4 *>(b + base);
  const float4 YM = *reinterpret_cast<const float4 *>(u + base - ys);
  const float4 YP = *reinterpret_cast<const float4 *>(u + base + ys);
  const float4 XM = *reinterpret_cast<const float4 *>(u + base - xs);
  const float4 XP = *reinterpret_cast<const float4 *>(u + base + xs);
  // the row neighbours beyond the warp's 128 cells: k4 - 1 for lane 0 (a ghost at k = -1 when
  // k4 == 0), k4 + 4 for lane 31 (a ghost at k = nz at the row's end).  Every lane loads (the
  // others a cell of the same lines), so the load issues with the float4 loads and costs no
  // second round trip.
  const float E = u[base + (lane == 31 ? 4 : -1)];
  float left = __shfl_up_sync(0xffffffffu, U.w, 1);
  float right = __shfl_down_sync(0xffffffffu, U.x, 1);
  if (lane == 0) left = E;
  if (lane == 31) right = E;
  float4 out = U;
  int k0, k1;
  float v0, v1;
  if (par == 0) {
    k0 = k4, k1 = k4 + 2;
    out.x = v0 = v4_update<float>(U.x, B.x, left, U.y, YM.x, YP.x, XM.x, XP.x, i, j, k0, nx, ny, nz, face_row, c);
    out.z = v1 = v4_update<float>(U.z, B.z, U.y, U.w, YM.z, YP.z, XM.z, XP.z, i, j, k1, nx, ny, nz, face_row, c);
  } else {
    k0 = k4 + 1, k1 = k4 + 3;
    out.y = v0 = v4_update<float>(U.y, B.y, U.x, U.z, YM.y, YP.y, XM.y, XP.y, i, j, k0, nx, ny, nz, face_row, c);
    out.w = v1 = v4_update<float>(U.w, B.w, U.z, right, YM.w, YP.w, XM.w, XP.w, i, j, k1, nx, ny, nz, face_row, c);
  }
  *reinterpret_cast<float4 *>(u + base) = out;
  if (face_row) {
    ge.emit(i, j, k0, v0);
    ge.emit(i, j, k1, v1);
    return;
  }
  // z-face ghosts of an interior row: a Dirichlet/Neumann ghost's source is the adjacent cell, a
  // periodic ghost's the cell on the opposite face
  const int row = base - k4;
  const int tn = ge.bc.type[FZ_NEG], tp = ge.bc.type[FZ_POS];
  if (k0 == 0) {
    if (tn == OCU_BC_DIRICHELET || tn == OCU_BC_NEUMANN) u[row - 1] = ge.template rule<FZ_NEG>(v0, ge.hz);
    if (tp == OCU_BC_PERIODIC) u[row + nz] = ge.template rule<FZ_POS>(v0, ge.hz);
  }
  if (k1 == nz - 1) {
    if (tp == OCU_BC_DIRICHELET || tp == OCU_BC_NEUMANN) u[row + nz] = ge.template rule<FZ_POS>(v1, ge.hz);
    if (tn == OCU_BC_PERIODIC) u[row - 1] = ge.template rule<FZ_NEG>(v1, ge.hz);
  }
}

template <typename T>
static bool launch_color_v4(T *, const T *, const ocu_layout &, int, const RelaxCoefD<T> &, const GhostEmit<T> &,
                            const T *, cudaStream_t) {
  return false;
}
template <>
bool launch_color_v4<float>(float *u, const float *b, const ocu_layout &L, int color, const RelaxCoefD<float> &c,
                            const GhostEmit<float> &ge, const float *, cudaStream_t s) {
  if (L.nz % 128 != 0 || L.allocated >= (1LL << 31) || L.shift % 4 != 0 || L.ystride % 4 != 0) return false;
  dim3 block(32, 4, 2), grid((L.nz + 127) / 128, (L.ny + 3) / 4, (L.nx + 1) / 2);
  launch_pdl(k_relax_color_v4, grid, block, 0, s, u, b, (int)L.xstride, (int)L.ystride, L.nx, L.ny, L.nz, color, c, ge);
  return true;
}

template <typename T>
ocu_status launch_relax_color_emit(T *u, const T *b, const ocu_layout &L, const T *diag, int color,
                                   const RelaxParams &p, double hx, double hy, double hz, cudaStream_t s) {
  const RelaxCoefD<T> c = make_relax_coef_d<T>(p);
  const int half = L.nz / 2;
  if (half == 0) return OCU_OK;
  dim3 block(half >= 32 ? 32 : (half >= 16 ? 16 : (half >= 8 ? 8 : 4)), 4, 2);
  block.y = 256 / (block.x * block.z) > 8 ? 8 : 256 / (block.x * block.z);
  dim3 grid((half + block.x - 1) / block.x, (L.ny + block.y - 1) / block.y, (L.nx + block.z - 1) / block.z);
  GhostEmit<T> ge{nullptr, L.xstride, L.ystride, L.nx, L.ny, L.nz, to_dev(p.bc), (T)hx, (T)hy, (T)hz};
  ge.p = u;
  if (launch_color_v4<T>(u, b, L, color, c, ge, diag, s)) return check_launch("k_relax_color_v4");
  const bool zfast = sizeof(T) == 8 && (long long)L.nx * L.ny * L.nz >= (1LL << 21);  // FP64, 128^3 and up
  if (L.allocated < (1LL << 31)) {
    if (zfast)
      launch_pdl(k_relax_color_emit<T, int, true>, grid, block, 0, s, u, b, (int)L.xstride, (int)L.ystride, L.nx,
                 L.ny, L.nz, color, c, diag, ge);
    else
      launch_pdl(k_relax_color_emit<T, int, false>, grid, block, 0, s, u, b, (int)L.xstride, (int)L.ystride, L.nx,
                 L.ny, L.nz, color, c, diag, ge);
  } else {
    launch_pdl(k_relax_color_emit<T, long long, false>, grid, block, 0, s, u, b, L.xstride, L.ystride, L.nx, L.ny,
               L.nz, color, c, diag, ge);
  }
  return check_launch("k_relax_color_emit");
}

// Prolongation + correction + ghost writes (devf.cu:94-197 then the level1 fill).
// EMIT = false compiles the ghost writes out (children that touch no face, or no fusable BCs).
template <typename T, bool EMIT, typename I = long long>
__device__ __forceinline__ void prolong_cell(const T *__restrict__ uc, I tc, I cx, I cy, T *__restrict__ uf, I f,
                                             I fxs, I fys, int ic, int jc, int kc, const GhostEmit<T> *ge) {
  const T w1 = (T)0.421875, w2 = (T)0.140625, w3 = (T)0.046875, w4 = (T)0.015625;
  const int i = 2 * ic + 1, j = 2 * jc + 1, k = 2 * kc + 1;
  // all eight fine values are loaded before the first store: the ghost writes go through
  // another pointer, so loads placed after a store could not be issued until it completed
  const T f000 = uf[f], f100 = uf[f - fxs], f010 = uf[f - fys];
  const T f001 = uf[f - 1];
  const T f110 = uf[f - fxs - fys], f101 = uf[f - fxs - 1], f011 = uf[f - fys - 1];
  const T f111 = uf[f - fxs - fys - 1];
  const T c000 = uc[tc];
  const T c0p0 = uc[tc + cy], c00p = uc[tc + 1], c0pp = uc[tc + cy + 1];
  const T c0m0 = uc[tc - cy], c00m = uc[tc - 1], c0mm = uc[tc - cy - 1];
  const T c0mp = uc[tc - cy + 1], c0pm = uc[tc + cy - 1];
  T v;
  {  // children on the +x side of the coarse centre (coarse plane x+1)
    const T cp00 = uc[tc + cx], cpp0 = uc[tc + cx + cy], cp0p = uc[tc + cx + 1];
    const T cppp = uc[tc + cx + cy + 1];
    const T cpm0 = uc[tc + cx - cy], cp0m = uc[tc + cx - 1], cpmm = uc[tc + cx - cy - 1];
    const T cppm = uc[tc + cx + cy - 1], cpmp = uc[tc + cx - cy + 1];
    v = f000 + w1 * c000 + w2 * (cp00 + c0p0 + c00p) + w3 * (cpp0 + cp0p + c0pp) + w4 * cppp;
    uf[f] = v; if (EMIT) ge->emit(i, j, k, v);
    v = f010 + w1 * c000 + w2 * (cp00 + c0m0 + c00p) + w3 * (cpm0 + cp0p + c0mp) + w4 * cpmp;
    uf[f - fys] = v; if (EMIT) ge->emit(i, j - 1, k, v);
    v = f001 + w1 * c000 + w2 * (cp00 + c0p0 + c00m) + w3 * (cpp0 + cp0m + c0pm) + w4 * cppm;
    uf[f - 1] = v; if (EMIT) ge->emit(i, j, k - 1, v);
    v = f011 + w1 * c000 + w2 * (cp00 + c0m0 + c00m) + w3 * (cpm0 + cp0m + c0mm) + w4 * cpmm;
    uf[f - fys - 1] = v; if (EMIT) ge->emit(i, j - 1, k - 1, v);
    // the -x child with (0,0) y/z offsets takes its corner weight from cppp, as the reference
    // kernel does (devf.cu:94-197)
    const T cm00 = uc[tc - cx], cmp0 = uc[tc - cx + cy], cm0p = uc[tc - cx + 1];
    v = f100 + w1 * c000 + w2 * (cm00 + c0p0 + c00p) + w3 * (cmp0 + cm0p + c0pp) + w4 * cppp;
    uf[f - fxs] = v; if (EMIT) ge->emit(i - 1, j, k, v);
  }
  {  // remaining children on the -x side (coarse plane x-1)
    const T cm00 = uc[tc - cx], cmm0 = uc[tc - cx - cy], cm0p = uc[tc - cx + 1];
    const T cm0m = uc[tc - cx - 1];
    const T cmmm = uc[tc - cx - cy - 1], cmp0 = uc[tc - cx + cy];
    const T cmpm = uc[tc - cx + cy - 1];
    const T cmmp = uc[tc - cx - cy + 1];
    v = f110 + w1 * c000 + w2 * (cm00 + c0m0 + c00p) + w3 * (cmm0 + cm0p + c0mp) + w4 * cmmp;
    uf[f - fxs - fys] = v; if (EMIT) ge->emit(i - 1, j - 1, k, v);
    v = f101 + w1 * c000 + w2 * (cm00 + c0p0 + c00m) + w3 * (cmp0 + cm0m + c0pm) + w4 * cmpm;
    uf[f - fxs - 1] = v; if (EMIT) ge->emit(i - 1, j, k - 1, v);
    v = f111 + w1 * c000 + w2 * (cm00 + c0m0 + c00m) + w3 * (cmm0 + cm0m + c0mm) + w4 * cmmm;
    uf[f - fxs - fys - 1] = v; if (EMIT) ge->emit(i - 1, j - 1, k - 1, v);
  }
}

template <typename T, typename I>
__global__ void __launch_bounds__(256, 4) k_prolong_emit(const T *__restrict__ uc, I cx, I cy, int cnx, int cny,
                                                         int cnz, T *__restrict__ uf, I fxs, I fys,
                                                         const __grid_constant__ GhostEmit<T> ge) {
  pdl_entry();
  const int kc = blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  const int ic = blockIdx.z;
  if (kc >= cnz || jc >= cny || ic >= cnx) return;
  const I tc = (I)ic * cx + (I)jc * cy + kc;
  const I f = (I)(2 * ic + 1) * fxs + (I)(2 * jc + 1) * fys + (2 * kc + 1);
  // only children on the fine grid's outer layer are ghost sources
  if (ic == 0 || ic == cnx - 1 || jc == 0 || jc == cny - 1 || kc == 0 || kc == cnz - 1)
    prolong_cell<T, true, I>(uc, tc, cx, cy, uf, f, fxs, fys, ic, jc, kc, &ge);
  else
    prolong_cell<T, false, I>(uc, tc, cx, cy, uf, f, fxs, fys, ic, jc, kc, nullptr);
}

// FP32 prolongation on float4 fine rows: a lane owns two adjacent coarse cells (kc = 2m, 2m+1) of
// a coarse row and writes their 16 children as four float4 fine-row segments (fine k = 4m..4m+3).
// The nine coarse rows (ic+-1, jc+-1) are read as float2 at k = 2m, 2m+1, with k = 2m-1 and 2m+2
// from the adjacent lanes.  Each child uses the same operand order as prolong_cell (including
// the corner weight of the (-1,0,0) child).  Coarse rows whose children touch a j or i face
// write every ghost of their children (GhostEmit); the others only have z-face ghosts, stored
// with the z rule.  cnz must be a multiple of 64.
template <typename T>
__device__ __forceinline__ T prolong_child(T f, T c000, T X, T Y, T Z, T XY, T XZ, T YZ, T XYZ) {
  const T w1 = (T)0.421875, w2 = (T)0.140625, w3 = (T)0.046875, w4 = (T)0.015625;
  return f + w1 * c000 + w2 * (X + Y + Z) + w3 * (XY + XZ + YZ) + w4 * XYZ;
}

// Ghosts of the 16 fine cells a thread of a face row wrote (re-read from u): every ghost rule,
// out of line so that the main body keeps its register budget.
template <typename T, int KN>
__device__ __noinline__ void prolong_row_ghosts(const GhostEmit<T> *ge, const T *uf, int fxs, int fys, int ic, int jc,
                                                int k0) {
  for (int dx = 0; dx < 2; dx++)
    for (int dy = 0; dy < 2; dy++) {
      const int fi = 2 * ic + 1 - dx, fj = 2 * jc + 1 - dy;
      for (int q = 0; q < KN; q++) ge->emit(fi, fj, k0 + q, uf[fi * fxs + fj * fys + k0 + q]);
    }
}

__global__ void __launch_bounds__(256, 4) k_prolong_v4(const float *__restrict__ uc, int cx, int cy, int cnx,
                                                       int cny, int cnz, float *__restrict__ uf, int fxs, int fys,
                                                       const __grid_constant__ GhostEmit<float> ge) {
  pdl_entry();
  const int lane = threadIdx.x;
  const int m = blockIdx.x * 32 + lane;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  // block row 0 takes the last coarse plane pair: both face planes (the slowest rows) run first
  const int bz = blockIdx.z == 0 ? gridDim.z - 1 : blockIdx.z - 1;
  const int ic = bz * blockDim.z + threadIdx.z;
  if (ic >= cnx || jc >= cny) return;  // whole warps (one coarse row each)
  const bool face = ic == 0 || ic == cnx - 1 || jc == 0 || jc == cny - 1;
  // coarse rows of the plane ic + di as c[dj+1][q], q = 0..3 for coarse k = 2m-1 .. 2m+2 (ghost
  // rows and planes included)
  auto load_plane = [&](int di, float (&c)[3][4]) {
#pragma unroll
    for (int dj = -1; dj <= 1; dj++) {
      const int base = (ic + di) * cx + (jc + dj) * cy + 2 * m;
      const float2 v = *reinterpret_cast<const float2 *>(uc + base);
      const float E = uc[base + (lane == 31 ? 2 : -1)];  // as in k_relax_color_v4: one load for all lanes
      float l = __shfl_up_sync(0xffffffffu, v.y, 1), r = __shfl_down_sync(0xffffffffu, v.x, 1);
      if (lane == 0) l = E;
      if (lane == 31) r = E;
      c[dj + 1][0] = l;
      c[dj + 1][1] = v.x;
      c[dj + 1][2] = v.y;
      c[dj + 1][3] = r;
    }
  };
  float c0[3][4], cs[3][4];
  // all 16 fine values first: loads placed after a store to uf could not be issued before it
  float4 FF[2][2];
#pragma unroll
  for (int dx = 0; dx < 2; dx++)
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
      FF[dx][dy] = *reinterpret_cast<const float4 *>(uf + (2 * ic + 1 - dx) * fxs + (2 * jc + 1 - dy) * fys + 4 * m);
  load_plane(0, c0);
  float cppp[2];  // corner weight of the (-x, +y, +z) children: coarse (ic+1, jc+1, kc+1)
  const int tn = ge.bc.type[FZ_NEG], tp = ge.bc.type[FZ_POS], fnz = 2 * cnz;
#pragma unroll
  for (int dx = 0; dx < 2; dx++) {  // dx = 0: fine row 2ic+1 (+x side); dx = 1: fine row 2ic (-x side)
    const int fi = 2 * ic + 1 - dx;
    const float4 *F = FF[dx];
    load_plane(dx ? -1 : 1, cs);
    if (dx == 0) {
      cppp[0] = cs[2][2];
      cppp[1] = cs[2][3];
    }
#pragma unroll
    for (int dy = 0; dy < 2; dy++) {
      const int sy = dy ? 0 : 2;  // neighbour row in c0/cs on the child's y side
      float out[4];
#pragma unroll
      for (int q = 0; q < 2; q++) {       // coarse cell kc = 2m + q, centre index q + 1
#pragma unroll
        for (int dz = 0; dz < 2; dz++) {  // dz = 0: fine k = 2kc+1 (+z side); dz = 1: 2kc (-z side)
          const int cq = q + 1, sz = dz ? q : q + 2, o = 2 * q + (dz ? 0 : 1);
          const float XYZ = (dx == 1 && dy == 0 && dz == 0) ? cppp[q] : cs[sy][sz];
          out[o] = prolong_child<float>((&F[dy].x)[o], c0[1][cq], cs[1][cq], c0[sy][cq], c0[1][sz], cs[sy][cq], cs[1][sz],
                                 c0[sy][sz], XYZ);
        }
      }
      const int fr = fi * fxs + (2 * jc + 1 - dy) * fys;  // fine row, k = 0
      *reinterpret_cast<float4 *>(uf + fr + 4 * m) = make_float4(out[0], out[1], out[2], out[3]);
      if (!face) {  // z-face ghosts of an interior fine row (GhostEmit writes exactly these there)
        if (m == 0) {
          if (tn == OCU_BC_DIRICHELET || tn == OCU_BC_NEUMANN) uf[fr - 1] = ge.template rule<FZ_NEG>(out[0], ge.hz);
          if (tp == OCU_BC_PERIODIC) uf[fr + fnz] = ge.template rule<FZ_POS>(out[0], ge.hz);
        }
        if (4 * m + 3 == fnz - 1) {
          if (tp == OCU_BC_DIRICHELET || tp == OCU_BC_NEUMANN) uf[fr + fnz] = ge.template rule<FZ_POS>(out[3], ge.hz);
          if (tn == OCU_BC_PERIODIC) uf[fr - 1] = ge.template rule<FZ_NEG>(out[3], ge.hz);
        }
      }
    }
  }
  if (face) prolong_row_ghosts<float, 4>(&ge, uf, fxs, fys, ic, jc, 4 * m);
}

// FP64 prolongation on double2 fine rows: a lane owns one coarse cell of a row (its 8 children
// are four double2 segments, fine k = 2kc, 2kc+1); coarse rows around it are scalar loads with
// the row neighbours from the adjacent lanes; same child sums, ghost writes and block order as
// k_prolong_v4.  cnz must be a multiple of 32.
__global__ void __launch_bounds__(256, 4) k_prolong_v2d(const double *__restrict__ uc, int cx, int cy, int cnx,
                                                        int cny, int cnz, double *__restrict__ uf, int fxs, int fys,
                                                        const __grid_constant__ GhostEmit<double> ge) {
  pdl_entry();
  const int lane = threadIdx.x;
  const int kc = blockIdx.x * 32 + lane;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  const int bz = blockIdx.z == 0 ? gridDim.z - 1 : blockIdx.z - 1;  // face planes first
  const int ic = bz * blockDim.z + threadIdx.z;
  if (ic >= cnx || jc >= cny) return;  // whole warps (one coarse row each)
  const bool face = ic == 0 || ic == cnx - 1 || jc == 0 || jc == cny - 1;
  // coarse rows of the plane ic + di as c[dj+1][q], q = 0..2 for coarse k = kc-1 .. kc+1
  auto load_plane = [&](int di, double (&c)[3][3]) {
#pragma unroll
    for (int dj = -1; dj <= 1; dj++) {
      const int base = (ic + di) * cx + (jc + dj) * cy + kc;
      const double v = uc[base];
      const double E = uc[base + (lane == 31 ? 1 : -1)];
      double l = __shfl_up_sync(0xffffffffu, v, 1), r = __shfl_down_sync(0xffffffffu, v, 1);
      if (lane == 0) l = E;
      if (lane == 31) r = E;
      c[dj + 1][0] = l;
      c[dj + 1][1] = v;
      c[dj + 1][2] = r;
    }
  };
  double c0[3][3], cs[3][3];
  double2 FF[2][2];  // all 8 fine values before the first store
#pragma unroll
  for (int dx = 0; dx < 2; dx++)
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
      FF[dx][dy] = *reinterpret_cast<const double2 *>(uf + (2 * ic + 1 - dx) * fxs + (2 * jc + 1 - dy) * fys + 2 * kc);
  load_plane(0, c0);
  double cppp = 0;  // corner weight of the (-x, +y, +z) child: coarse (ic+1, jc+1, kc+1)
  const int tn = ge.bc.type[FZ_NEG], tp = ge.bc.type[FZ_POS], fnz = 2 * cnz;
#pragma unroll
  for (int dx = 0; dx < 2; dx++) {  // dx = 0: fine row 2ic+1 (+x side); dx = 1: fine row 2ic (-x side)
    const int fi = 2 * ic + 1 - dx;
    const double2 *F = FF[dx];
    load_plane(dx ? -1 : 1, cs);
    if (dx == 0) cppp = cs[2][2];
#pragma unroll
    for (int dy = 0; dy < 2; dy++) {
      const int sy = dy ? 0 : 2;
      double out[2];
#pragma unroll
      for (int dz = 0; dz < 2; dz++) {  // dz = 0: fine k = 2kc+1 (+z side, .y); dz = 1: 2kc (-z side, .x)
        const int sz = dz ? 0 : 2, o = dz ? 0 : 1;
        const double XYZ = (dx == 1 && dy == 0 && dz == 0) ? cppp : cs[sy][sz];
        out[o] = prolong_child<double>(o ? F[dy].y : F[dy].x, c0[1][1], cs[1][1], c0[sy][1], c0[1][sz], cs[sy][1],
                                       cs[1][sz], c0[sy][sz], XYZ);
      }
      const int fr = fi * fxs + (2 * jc + 1 - dy) * fys;  // fine row, k = 0
      *reinterpret_cast<double2 *>(uf + fr + 2 * kc) = make_double2(out[0], out[1]);
      if (!face) {  // z-face ghosts of an interior fine row
        if (kc == 0) {
          if (tn == OCU_BC_DIRICHELET || tn == OCU_BC_NEUMANN) uf[fr - 1] = ge.template rule<FZ_NEG>(out[0], ge.hz);
          if (tp == OCU_BC_PERIODIC) uf[fr + fnz] = ge.template rule<FZ_POS>(out[0], ge.hz);
        }
        if (2 * kc + 1 == fnz - 1) {
          if (tp == OCU_BC_DIRICHELET || tp == OCU_BC_NEUMANN) uf[fr + fnz] = ge.template rule<FZ_POS>(out[1], ge.hz);
          if (tn == OCU_BC_PERIODIC) uf[fr - 1] = ge.template rule<FZ_NEG>(out[1], ge.hz);
        }
      }
    }
  }
  if (face) prolong_row_ghosts<double, 2>(&ge, uf, fxs, fys, ic, jc, 2 * kc);
}

// coarse levels up to this many cells prolong with one thread per fine cell
constexpr long long kProlongFineCells = 32768;

// Prolongation with one thread per FINE cell: the child's coarse octant (eight values), the
// same sum and corner rule as prolong_cell, then its ghosts.  For the small levels, whose
// launches are latency-bound: a thread's chain is one child instead of eight children and
// their ghost writes.
template <typename T>
__global__ void __launch_bounds__(256) k_prolong_fine(const T *__restrict__ uc, int cx, int cy, int cnx, int cny,
                                                      int cnz, T *__restrict__ uf, int fxs, int fys,
                                                      const __grid_constant__ GhostEmit<T> ge) {
  pdl_entry();
  const int fk = blockIdx.x * blockDim.x + threadIdx.x;
  const int fj = blockIdx.y * blockDim.y + threadIdx.y;
  const int bz = blockIdx.z == 0 ? gridDim.z - 1 : blockIdx.z - 1;  // face planes first
  const int fi = bz * blockDim.z + threadIdx.z;
  if (fk >= 2 * cnz || fj >= 2 * cny || fi >= 2 * cnx) return;
  const int dx = 1 - (fi & 1), dy = 1 - (fj & 1), dz = 1 - (fk & 1);  // 1: the child on the parent's - side
  const int sx = dx ? -cx : cx, sy = dy ? -cy : cy, sz = dz ? -1 : 1;
  const int tc = (fi >> 1) * cx + (fj >> 1) * cy + (fk >> 1);
  const int f = fi * fxs + fj * fys + fk;
  const T fv = uf[f];
  const T c000 = uc[tc], X = uc[tc + sx], Y = uc[tc + sy], Z = uc[tc + sz];
  const T XY = uc[tc + sx + sy], XZ = uc[tc + sx + sz], YZ = uc[tc + sy + sz];
  // the (-x, +y, +z) child takes its corner weight from (+1, +1, +1), as prolong_cell does
  const T XYZ = (dx == 1 && dy == 0 && dz == 0) ? uc[tc + cx + cy + 1] : uc[tc + sx + sy + sz];
  const T v = prolong_child<T>(fv, c000, X, Y, Z, XY, XZ, YZ, XYZ);
  uf[f] = v;
  ge.emit(fi, fj, fk, v);
}

template <typename T>
ocu_status launch_prolong_emit(const T *uc, const ocu_layout &Lc, T *uf, const ocu_layout &Lf,
                               const ocu_bc_set &bc_fine, double hx, double hy, double hz, cudaStream_t s) {
  dim3 block(Lc.nz >= 32 ? 32 : 16, 8);
  dim3 grid((Lc.nz + block.x - 1) / block.x, (Lc.ny + block.y - 1) / block.y, Lc.nx);
  GhostEmit<T> ge{uf, Lf.xstride, Lf.ystride, Lf.nx, Lf.ny, Lf.nz, to_dev(bc_fine), (T)hx, (T)hy, (T)hz};
  // one thread per fine cell on the small levels: FP32 up to 64^3 coarse cells (measured faster
  // than the float4 kernel there, 13.4 against 16.7 us into 128^3), FP64 up to 32^3 where the
  // double2 kernel does not apply (it is faster into 128^3: 12.6 against 14.2 us)
  const long long ccells = (long long)Lc.nx * Lc.ny * Lc.nz;
  auto launch_fine = [&]() {
    const int fz = 2 * Lc.nz;
    dim3 bf(fz >= 32 ? 32 : (fz >= 16 ? 16 : (fz >= 8 ? 8 : 4)), 4, 2);
    bf.y = 256 / (bf.x * bf.z) > 8 ? 8 : 256 / (bf.x * bf.z);
    dim3 gf((fz + bf.x - 1) / bf.x, (2 * Lc.ny + bf.y - 1) / bf.y, (2 * Lc.nx + bf.z - 1) / bf.z);
    launch_pdl(k_prolong_fine<T>, gf, bf, 0, s, uc, (int)Lc.xstride, (int)Lc.ystride, Lc.nx, Lc.ny, Lc.nz, uf,
               (int)Lf.xstride, (int)Lf.ystride, ge);
    return check_launch("k_prolong_fine");
  };
  const bool fine_ok = Lf.allocated < (1LL << 31);
  if (sizeof(T) == 4 && fine_ok && ccells <= 8 * kProlongFineCells) return launch_fine();
  if (sizeof(T) == 4 && Lc.nz % 64 == 0 && Lf.allocated < (1LL << 31) && Lc.shift % 2 == 0 && Lf.shift % 4 == 0 &&
      Lc.ystride % 2 == 0 && Lf.ystride % 4 == 0) {
    dim3 b4(32, 4, 2), g4(Lc.nz / 64, (Lc.ny + 3) / 4, (Lc.nx + 1) / 2);
    launch_pdl(k_prolong_v4, g4, b4, 0, s, (const float *)uc, (int)Lc.xstride, (int)Lc.ystride, Lc.nx, Lc.ny, Lc.nz,
               (float *)uf, (int)Lf.xstride, (int)Lf.ystride, *reinterpret_cast<const GhostEmit<float> *>(&ge));
    return check_launch("k_prolong_v4");
  }
  if (sizeof(T) == 8 && Lc.nz % 32 == 0 && Lf.allocated < (1LL << 31) && Lf.shift % 2 == 0 &&
      Lf.ystride % 2 == 0) {
    dim3 b2(32, 4, 2), g2(Lc.nz / 32, (Lc.ny + 3) / 4, (Lc.nx + 1) / 2);
    launch_pdl(k_prolong_v2d, g2, b2, 0, s, (const double *)uc, (int)Lc.xstride, (int)Lc.ystride, Lc.nx, Lc.ny, Lc.nz,
               (double *)uf, (int)Lf.xstride, (int)Lf.ystride, *reinterpret_cast<const GhostEmit<double> *>(&ge));
    return check_launch("k_prolong_v2d");
  }
  if (fine_ok && ccells <= kProlongFineCells) return launch_fine();
  if (Lf.allocated < (1LL << 31) && Lc.allocated < (1LL << 31))
    launch_pdl(k_prolong_emit<T, int>, grid, block, 0, s, uc, (int)Lc.xstride, (int)Lc.ystride, Lc.nx, Lc.ny, Lc.nz, uf,
               (int)Lf.xstride, (int)Lf.ystride, ge);
  else
    launch_pdl(k_prolong_emit<T, long long>, grid, block, 0, s, uc, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, uf,
               Lf.xstride, Lf.ystride, ge);
  return check_launch("k_prolong_emit");
}

// ------------------------------------------------------------------------------------------
// Residual helpers
// ------------------------------------------------------------------------------------------
// Fold one 64-wide chunk of a fine row into the lane accumulators in reference order:
// this lane holds r at k = base + 2*lane (+1); virtual lane t needs k = base + t and
// base + 32 + t, held by lanes t/2 and 16 + t/2.
template <typename T>
__device__ __forceinline__ void fold_chunk(T e0, T e1, int base, int nz, int lane, T &acc2, T &accinf,
                                           bool want2, bool wantinf) {
  const int src1 = lane >> 1, src2 = 16 + (lane >> 1);
  const T a0 = __shfl_sync(0xffffffffu, e0, src1), a1 = __shfl_sync(0xffffffffu, e1, src1);
  const T b0 = __shfl_sync(0xffffffffu, e0, src2), b1 = __shfl_sync(0xffffffffu, e1, src2);
  const T x1 = (lane & 1) ? a1 : a0;
  const T x2 = (lane & 1) ? b1 : b0;
  if (base + lane < nz) {
    if (want2) acc2 = x1 * x1 + acc2;
    if (wantinf) accinf = fmax(fabs(x1), accinf);
  }
  if (base + 32 + lane < nz) {
    if (want2) acc2 = x2 * x2 + acc2;
    if (wantinf) accinf = fmax(fabs(x2), accinf);
  }
}

template <typename T>
__device__ __forceinline__ T warp_tree(T v, bool is_max) {
  for (int o = 16; o > 0; o >>= 1) {
    const T other = __shfl_down_sync(0xffffffffu, v, o);
    v = is_max ? fmax(v, other) : v + other;
  }
  return v;
}

template <typename T> struct Vec2T;
template <> struct Vec2T<float> { using type = float2; };
template <> struct Vec2T<double> { using type = double2; };

template <typename T>
__device__ __forceinline__ T residual_pt(T bv, T uc, T zm, T zp, T ym, T yp, T xm, T xp, const ResCoefT<T> &c) {
  return bv - (c.fzh * (zm + zp) + c.fyh * (ym + yp) + c.fxh * (xm + xp) - c.dg * uc);
}

// Residual over one fine row per warp (chunks of 64 along k): optional outputs r (T), r as
// float (the refinement solver's FP32 right-hand side), and per-row norm partials.
template <typename T, bool VEC>
__global__ void __launch_bounds__(256) k_residual_rows(const T *__restrict__ u, const T *__restrict__ b,
                                                       T *__restrict__ r, float *__restrict__ r32, long long xs,
                                                       long long ys, int nx, int ny, int nz, ResCoefT<T> c,
                                                       T *__restrict__ rows2, T *__restrict__ rowsinf) {
  pdl_entry();
  const int lane = threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (j >= ny) return;  // whole warp exits together
  const bool want2 = rows2 != nullptr, wantinf = rowsinf != nullptr;
  T acc2 = 0, accinf = 0;
  const long long row = (long long)i * xs + (long long)j * ys;
  if (VEC) {  // nz even, rows 16-byte aligned: a lane's two cells and their neighbours as 2-wide loads
    using V = typename Vec2T<T>::type;
    for (int base = 0; base < nz; base += 64) {
      const int k0 = base + 2 * lane;
      T e0 = 0, e1 = 0;
      if (k0 < nz) {
        const long long id = row + k0;
        const V U = *reinterpret_cast<const V *>(u + id), B = *reinterpret_cast<const V *>(b + id);
        const V YM = *reinterpret_cast<const V *>(u + id - ys), YP = *reinterpret_cast<const V *>(u + id + ys);
        const V XM = *reinterpret_cast<const V *>(u + id - xs), XP = *reinterpret_cast<const V *>(u + id + xs);
        const T L = u[id - 1], R = u[id + 2];
        e0 = residual_pt<T>(B.x, U.x, L, U.y, YM.x, YP.x, XM.x, XP.x, c);
        e1 = residual_pt<T>(B.y, U.y, U.x, R, YM.y, YP.y, XM.y, XP.y, c);
        if (r) {
          V o;
          o.x = e0;
          o.y = e1;
          *reinterpret_cast<V *>(r + id) = o;
        }
        if (r32) *reinterpret_cast<float2 *>(r32 + id) = make_float2((float)e0, (float)e1);
      }
      if (want2 || wantinf) fold_chunk<T>(e0, e1, base, nz, lane, acc2, accinf, want2, wantinf);
    }
  } else {
  for (int base = 0; base < nz; base += 64) {
    const int k0 = base + 2 * lane;
    T e0 = 0, e1 = 0;
    if (k0 < nz) {
      e0 = residual_at<T>(u, b, row + k0, xs, ys, c);
      if (r) r[row + k0] = e0;
      if (r32) r32[row + k0] = (float)e0;
    }
    if (k0 + 1 < nz) {
      e1 = residual_at<T>(u, b, row + k0 + 1, xs, ys, c);
      if (r) r[row + k0 + 1] = e1;
      if (r32) r32[row + k0 + 1] = (float)e1;
    }
    if (want2 || wantinf) fold_chunk<T>(e0, e1, base, nz, lane, acc2, accinf, want2, wantinf);
  }
  }
  if (want2) {
    const T v = warp_tree<T>(acc2, false);
    if (lane == 0) rows2[(long long)i * ny + j] = v;
  }
  if (wantinf) {
    const T v = warp_tree<T>(accinf, true);
    if (lane == 0) rowsinf[(long long)i * ny + j] = v;
  }
}

// Residual at the 8 children of each coarse cell + restriction, one coarse row per warp.
// The children's residuals are never stored; norm partials (level 0 only) fold the 4 fine rows
// (2ic+di, 2jc+dj) of the warp.
template <typename T, bool NORM>
__global__ void __launch_bounds__(256) k_residual_restrict(const T *__restrict__ u, const T *__restrict__ b,
                                                           long long xs, long long ys, int nx, int ny, int nz,
                                                           ResCoefT<T> c, T *__restrict__ bc_, long long bxs,
                                                           long long bys, int cnx, int cny, int cnz,
                                                           T *__restrict__ rows2, T *__restrict__ rowsinf, T *__restrict__ zero_u,
    long long zero_n) {
  pdl_entry();
  if (zero_u) {  // the coarser level's clear (its whole buffer, as a memset), nothing here reads it
    const long long nthreads = (long long)gridDim.x * gridDim.y * gridDim.z * blockDim.x * blockDim.y;
    const long long tid = ((long long)(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) *
                              (blockDim.x * blockDim.y) + threadIdx.y * blockDim.x + threadIdx.x;
    for (long long q = tid; q < zero_n; q += nthreads) zero_u[q] = (T)0;
  }
  const int lane = threadIdx.x;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  const int ic = blockIdx.z;
  if (jc >= cny) return;
  const bool want2 = NORM && rows2 != nullptr, wantinf = NORM && rowsinf != nullptr;
  T acc2[4] = {0, 0, 0, 0}, accinf[4] = {0, 0, 0, 0};
  const long long frow = (long long)(2 * ic) * xs + (long long)(2 * jc) * ys;
  // with norms a warp walks its whole row (the fold runs along k); without, one 32-cell chunk
  const int cfirst = NORM ? 0 : blockIdx.x * 32, cend = NORM ? cnz : min(cfirst + 32, cnz);
  for (int cbase = cfirst; cbase < cend; cbase += 32) {
    const int kc = cbase + lane;
    T r[8];
    if (kc < cnz) {
      const long long ri = frow + 2 * kc;
      r[0] = residual_at<T>(u, b, ri, xs, ys, c);
      r[1] = residual_at<T>(u, b, ri + 1, xs, ys, c);
      r[2] = residual_at<T>(u, b, ri + ys, xs, ys, c);
      r[3] = residual_at<T>(u, b, ri + 1 + ys, xs, ys, c);
      r[4] = residual_at<T>(u, b, ri + xs, xs, ys, c);
      r[5] = residual_at<T>(u, b, ri + 1 + xs, xs, ys, c);
      r[6] = residual_at<T>(u, b, ri + ys + xs, xs, ys, c);
      r[7] = residual_at<T>(u, b, ri + 1 + ys + xs, xs, ys, c);
      bc_[(long long)ic * bxs + (long long)jc * bys + kc] =
          (T)0.125 * (r[0] + r[1] + r[2] + r[3] + r[4] + r[5] + r[6] + r[7]);
    } else {
#pragma unroll
      for (int q = 0; q < 8; q++) r[q] = 0;
    }
    if (NORM && (want2 || wantinf)) {
      // fine rows: (di,dj) = (0,0): r0,r1 ; (0,1): r2,r3 ; (1,0): r4,r5 ; (1,1): r6,r7
#pragma unroll
      for (int q = 0; q < 4; q++)
        fold_chunk<T>(r[2 * q], r[2 * q + 1], 2 * cbase, nz, lane, acc2[q], accinf[q], want2, wantinf);
    }
  }
  if (NORM) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * ic + (q >> 1), j = 2 * jc + (q & 1);
      if (want2) {
        const T v = warp_tree<T>(acc2[q], false);
        if (lane == 0) rows2[(long long)i * ny + j] = v;
      }
      if (wantinf) {
        const T v = warp_tree<T>(accinf[q], true);
        if (lane == 0) rowsinf[(long long)i * ny + j] = v;
      }
    }
  }
}

// The same with 2-wide vector loads: a lane's two children of a fine row are one float2/double2,
// and so are their neighbours in the rows j-1 / j+2 and planes i-1 / i+2; the row neighbours
// k-1 and k+2 are scalar loads of the same lines.  24 load instructions per coarse cell instead
// of 64; each residual is residual_at's expression on the same operands.
template <typename T, bool NORM>
__global__ void __launch_bounds__(256) k_residual_restrict_v2(const T *__restrict__ u, const T *__restrict__ b,
                                                              long long xs, long long ys, int nx, int ny, int nz,
                                                              ResCoefT<T> c, T *__restrict__ bc_, long long bxs,
                                                              long long bys, int cnx, int cny, int cnz,
                                                              T *__restrict__ rows2, T *__restrict__ rowsinf, T *__restrict__ zero_u,
    long long zero_n) {
  using V = typename Vec2T<T>::type;
  pdl_entry();
  if (zero_u) {  // the coarser level's clear (its whole buffer, as a memset), nothing here reads it
    const long long nthreads = (long long)gridDim.x * gridDim.y * gridDim.z * blockDim.x * blockDim.y;
    const long long tid = ((long long)(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) *
                              (blockDim.x * blockDim.y) + threadIdx.y * blockDim.x + threadIdx.x;
    for (long long q = tid; q < zero_n; q += nthreads) zero_u[q] = (T)0;
  }
  const int lane = threadIdx.x;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  const int ic = blockIdx.z;
  if (jc >= cny) return;
  const bool want2 = NORM && rows2 != nullptr, wantinf = NORM && rowsinf != nullptr;
  T acc2[4] = {0, 0, 0, 0}, accinf[4] = {0, 0, 0, 0};
  const long long f00 = (long long)(2 * ic) * xs + (long long)(2 * jc) * ys;
  // with norms a warp walks its whole row (the fold runs along k); without, one 32-cell chunk
  const int cfirst = NORM ? 0 : blockIdx.x * 32, cend = NORM ? cnz : min(cfirst + 32, cnz);
  for (int cbase = cfirst; cbase < cend; cbase += 32) {
    const int kc = cbase + lane;
    const bool act = kc < cnz;
    const long long kk = 2 * (act ? kc : cnz - 1);  // lanes past the row end read the last pair
    V U[2][2], B[2][2], Yo[2][2], Xo[2][2];
    T Lz[2][2], Rz[2][2];
#pragma unroll
    for (int di = 0; di < 2; di++)
#pragma unroll
      for (int dj = 0; dj < 2; dj++) {
        const long long row = f00 + di * xs + dj * ys + kk;
        U[di][dj] = *reinterpret_cast<const V *>(u + row);
        B[di][dj] = *reinterpret_cast<const V *>(b + row);
        Yo[di][dj] = *reinterpret_cast<const V *>(u + row + (dj ? ys : -ys));  // rows 2jc-1 / 2jc+2
        Xo[di][dj] = *reinterpret_cast<const V *>(u + row + (di ? xs : -xs));  // planes 2ic-1 / 2ic+2
        Lz[di][dj] = u[row - 1];
        Rz[di][dj] = u[row + 2];
      }
    T r[8];
#pragma unroll
    for (int di = 0; di < 2; di++)
#pragma unroll
      for (int dj = 0; dj < 2; dj++)
#pragma unroll
        for (int dk = 0; dk < 2; dk++) {
          const V &uc = U[di][dj];
          const T ucv = dk ? uc.y : uc.x, bv = dk ? B[di][dj].y : B[di][dj].x;
          const T zm = dk ? uc.x : Lz[di][dj], zp = dk ? Rz[di][dj] : uc.y;
          const V &ymv = dj ? U[di][0] : Yo[di][0], &ypv = dj ? Yo[di][1] : U[di][1];
          const V &xmv = di ? U[0][dj] : Xo[0][dj], &xpv = di ? Xo[1][dj] : U[1][dj];
          const T ym = dk ? ymv.y : ymv.x, yp = dk ? ypv.y : ypv.x;
          const T xm = dk ? xmv.y : xmv.x, xp = dk ? xpv.y : xpv.x;
          r[4 * di + 2 * dj + dk] = act ? residual_pt<T>(bv, ucv, zm, zp, ym, yp, xm, xp, c) : (T)0;
        }
    if (act)
      bc_[(long long)ic * bxs + (long long)jc * bys + kc] =
          (T)0.125 * (r[0] + r[1] + r[2] + r[3] + r[4] + r[5] + r[6] + r[7]);
    if (NORM && (want2 || wantinf)) {
#pragma unroll
      for (int q = 0; q < 4; q++)
        fold_chunk<T>(r[2 * q], r[2 * q + 1], 2 * cbase, nz, lane, acc2[q], accinf[q], want2, wantinf);
    }
  }
  if (NORM) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * ic + (q >> 1), j = 2 * jc + (q & 1);
      if (want2) {
        const T v = warp_tree<T>(acc2[q], false);
        if (lane == 0) rows2[(long long)i * ny + j] = v;
      }
      if (wantinf) {
        const T v = warp_tree<T>(accinf[q], true);
        if (lane == 0) rowsinf[(long long)i * ny + j] = v;
      }
    }
  }
}

// Coarse levels up to this many cells (16^3) restrict with one thread per fine cell.  Measured
// at 256^3 (mixed solve, one box, both builds): 4.84 ms with this bound against 4.85 ms at 32^3
// and 4.92 ms at 64^3; at 8^3 no better than 32^3.
constexpr long long kRestrictFineCells = 4096;

// Residual + restriction for the small levels, without norms: eight lanes per coarse cell, one
// child each; the group's first lane gathers the eight residuals by shuffles and sums them in
// the per-operation kernels' order.  Short per-thread chains for latency-bound launches.
template <typename T>
__global__ void __launch_bounds__(256) k_residual_restrict_fine(const T *__restrict__ u, const T *__restrict__ b,
                                                                int xs, int ys, ResCoefT<T> c, T *__restrict__ bc_,
                                                                int bxs, int bys, int cnx, int cny, int cnz,
                                                                T *__restrict__ zero_u, long long zero_n) {
  pdl_entry();
  if (zero_u) {  // the coarser level's clear (its whole buffer, as a memset), nothing here reads it
    const long long nthreads = (long long)gridDim.x * gridDim.y * gridDim.z * blockDim.x;
    const long long tid = ((long long)(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * blockDim.x +
                          threadIdx.x;
    for (long long q = tid; q < zero_n; q += nthreads) zero_u[q] = (T)0;
  }
  const int child = threadIdx.x & 7;
  const int kc = blockIdx.x * (blockDim.x >> 3) + (threadIdx.x >> 3);
  const int jc = blockIdx.y, ic = blockIdx.z;
  const bool act = kc < cnz;
  const int di = child >> 2, dj = (child >> 1) & 1, dk = child & 1;
  const long long id = (long long)(2 * ic + di) * xs + (long long)(2 * jc + dj) * ys + 2 * (act ? kc : 0) + dk;
  const T r = residual_at<T>(u, b, id, xs, ys, c);
  // gather the group's residuals in child order r0..r7 = (0,0,0), (0,0,1), (0,1,0), ... (1,1,1)
  const int g = threadIdx.x & 31 & ~7;
  T rr[8];
#pragma unroll
  for (int n = 0; n < 8; n++) rr[n] = __shfl_sync(0xffffffffu, r, g + n);
  if (act && child == 0)
    bc_[(long long)ic * bxs + (long long)jc * bys + kc] =
        (T)0.125 * (rr[0] + rr[1] + rr[2] + rr[3] + rr[4] + rr[5] + rr[6] + rr[7]);
}

// 256-wide fold of row values (grid1dops.cu:33-115), one launch: block b folds rows
// [256b, 256b+256), the last block folds the block partials.  Writes the T result as double.
template <typename T>
__global__ void __launch_bounds__(256) k_fold_rows(const T *__restrict__ rows, long long nrows, int is_max,
                                                   T *partial, unsigned *counter, double *result) {
  pdl_entry();
  __shared__ T sh[256];
  __shared__ bool last;
  const long long idx = (long long)blockIdx.x * 256 + threadIdx.x;
  sh[threadIdx.x] = idx < nrows ? rows[idx] : (T)0;
  __syncthreads();
  for (int stride = 128; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride)
      sh[threadIdx.x] = is_max ? fmax(sh[threadIdx.x], sh[threadIdx.x + stride]) : sh[threadIdx.x] + sh[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = sh[0];
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  volatile T *vp = partial;
  long long count = gridDim.x;
  while (count > 1) {
    const long long nb = (count + 255) / 256;
    for (long long bb = 0; bb < nb; bb++) {
      const long long q = bb * 256 + threadIdx.x;
      sh[threadIdx.x] = q < count ? vp[q] : (T)0;
      __syncthreads();
      for (int stride = 128; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride)
          sh[threadIdx.x] = is_max ? fmax(sh[threadIdx.x], sh[threadIdx.x + stride]) : sh[threadIdx.x] + sh[threadIdx.x + stride];
        __syncthreads();
      }
      if (threadIdx.x == 0) vp[bb] = sh[0];
      __syncthreads();
    }
    count = nb;
  }
  if (threadIdx.x == 0) {
    *result = (double)vp[0];
    *counter = 0;
  }
}

template <typename T>
static ResCoefT<T> res_coef(double h, double fx, double fy, double fz) {
  ResCoefT<T> c;
  c.fxh = (T)(fx / (h * h));
  c.fyh = (T)(fy / (h * h));
  c.fzh = (T)(fz / (h * h));
  c.dg = (T)(2 * (fx + fy + fz) / (h * h));
  return c;
}

template <typename T>
ocu_status launch_residual_rows(const T *u, const T *b, T *r, float *r32, const ocu_layout &L, double h, double fx,
                                double fy, double fz, T *rows2, T *rowsinf, cudaStream_t s) {
  dim3 block(32, 8), grid(1, (L.ny + 7) / 8, L.nx);
  // the 2-wide path needs even rows starting on 2-element boundaries (r32 shares the layout)
  if (L.nz % 2 == 0 && L.shift % 2 == 0 && L.xstride % 2 == 0 && L.ystride % 2 == 0)
    launch_pdl(k_residual_rows<T, true>, grid, block, 0, s, u, b, r, r32, L.xstride, L.ystride, L.nx, L.ny, L.nz,
               res_coef<T>(h, fx, fy, fz), rows2, rowsinf);
  else
    launch_pdl(k_residual_rows<T, false>, grid, block, 0, s, u, b, r, r32, L.xstride, L.ystride, L.nx, L.ny, L.nz,
               res_coef<T>(h, fx, fy, fz), rows2, rowsinf);
  return check_launch("k_residual_rows");
}

template <typename T>
ocu_status launch_residual_restrict(const T *u, const T *b, const ocu_layout &Lf, T *bc_, const ocu_layout &Lc,
                                    double h, double fx, double fy, double fz, T *rows2, T *rowsinf, cudaStream_t s,
                                    T *zero_u, long long zero_n) {
  dim3 block(32, 8), grid(1, (Lc.ny + 7) / 8, Lc.nx);
  const ResCoefT<T> c = res_coef<T>(h, fx, fy, fz);
  if (!rows2 && !rowsinf && (long long)Lc.nx * Lc.ny * Lc.nz <= kRestrictFineCells && Lf.allocated < (1LL << 31) &&
      Lc.allocated < (1LL << 31)) {
    const int per_block = Lc.nz >= 32 ? 32 : (Lc.nz >= 16 ? 16 : (Lc.nz >= 8 ? 8 : 4));  // coarse cells
    dim3 gf((Lc.nz + per_block - 1) / per_block, Lc.ny, Lc.nx);
    launch_pdl(k_residual_restrict_fine<T>, gf, dim3(8 * per_block), 0, s, u, b, (int)Lf.xstride, (int)Lf.ystride, c,
               bc_, (int)Lc.xstride, (int)Lc.ystride, Lc.nx, Lc.ny, Lc.nz, zero_u, zero_n);
    return check_launch("k_residual_restrict_fine");
  }
  if (sizeof(T) == 4 && Lf.shift % 2 == 0 && Lf.xstride % 2 == 0 && Lf.ystride % 2 == 0 && Lf.nz == 2 * Lc.nz) {
    if (rows2 || rowsinf) {
      launch_pdl(k_residual_restrict_v2<T, true>, grid, block, 0, s, u, b, Lf.xstride, Lf.ystride, Lf.nx, Lf.ny, Lf.nz,
                 c, bc_, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, rows2, rowsinf, zero_u, zero_n);
    } else {
      dim3 gridc((Lc.nz + 31) / 32, (Lc.ny + 7) / 8, Lc.nx);
      launch_pdl(k_residual_restrict_v2<T, false>, gridc, block, 0, s, u, b, Lf.xstride, Lf.ystride, Lf.nx, Lf.ny,
                 Lf.nz, c, bc_, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, nullptr, nullptr, zero_u, zero_n);
    }
    return check_launch("k_residual_restrict_v2");
  }
  if (rows2 || rowsinf) {
    launch_pdl(k_residual_restrict<T, true>, grid, block, 0, s, u, b, Lf.xstride, Lf.ystride, Lf.nx, Lf.ny, Lf.nz, c,
               bc_, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, rows2, rowsinf, zero_u, zero_n);
  } else {
    dim3 gridc((Lc.nz + 31) / 32, (Lc.ny + 7) / 8, Lc.nx);
    launch_pdl(k_residual_restrict<T, false>, gridc, block, 0, s, u, b, Lf.xstride, Lf.ystride, Lf.nx, Lf.ny, Lf.nz, c,
               bc_, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, nullptr, nullptr, zero_u, zero_n);
  }
  return check_launch("k_residual_restrict");
}

template <typename T>
ocu_status launch_fold_rows(const T *rows, long long nrows, bool is_max, void *scratch, double *result,
                            cudaStream_t s) {
  const long long blocks = (nrows + 255) / 256;
  unsigned *counter = reinterpret_cast<unsigned *>(scratch);
  T *partial = reinterpret_cast<T *>(reinterpret_cast<char *>(scratch) + 64);
  launch_pdl(k_fold_rows<T>, (unsigned)blocks, 256, 0, s, rows, nrows, is_max ? 1 : 0, partial, counter, result);
  return check_launch("k_fold_rows");
}

// ------------------------------------------------------------------------------------------
// Single-CTA coarse tail: levels s..L-1 of one V-cycle (down: relax nu1, clear, residual +
// restrict; coarsest: relax with the host routine's arithmetic; up: prolong + ghosts, relax
// nu2), phases separated by __syncthreads.  Identical operation sequence and arithmetic to the
// per-level kernels.
// ------------------------------------------------------------------------------------------
// The tail's phases are separate (not inlined) functions: the kernel runs each code path only a
// few times per launch, so one shared copy of every phase keeps its instruction footprint (and
// the cold instruction fetches that dominated it) small.
// Phases take their cells from t0 in steps of nt (threadIdx.x / blockDim.x).
template <typename T>
__device__ __noinline__ void tail_relax(const TailLevel<T> &lv, int iterations, int order, int t0, int nt) {
  GhostEmit<T> ge{lv.u, lv.xs, lv.ys, lv.nx, lv.ny, lv.nz, lv.bc, lv.hx, lv.hy, lv.hz};
  if (order == 2) {
    if (iterations % 2 == 1) iterations++;
    if (iterations < 4) iterations = 4;
  }
  const int half = lv.nz / 2;
  const int nwork = lv.nx * lv.ny * half;
  for (int it = 0; it < iterations; it++) {
    for (int rb = 0; rb < 2; rb++) {
      int color = rb;
      if (order == 1 || (order == 2 && it >= iterations / 2)) color = !rb;
      for (int q = t0; q < nwork; q += nt) {
        const int i = q / (lv.ny * half), rem = q % (lv.ny * half), j = rem / half, t = rem % half;
        const int k = 2 * t + ((i + j + color) & 1);
        const long long id = (long long)i * lv.xs + (long long)j * lv.ys + k;
        const T nv = relax_point<T>(lv.u, lv.b, id, lv.xs, lv.ys, i, j, k, lv.nx, lv.ny, lv.nz, lv.rc, nullptr);
        lv.u[id] = nv;
        if (lv.emit_ok) ge.emit(i, j, k, nv);
      }
      __syncthreads();
      // without fused ghost writes: refresh between colours when periodic, else after both
      // (sol_mgpressure3ddev.cu:235-241)
      if (!lv.emit_ok && (lv.periodic || rb == 1)) {
        level1_fill_block<T>(lv.u, lv.xs, lv.ys, lv.nx, lv.ny, lv.nz, lv.bc, lv.hx, lv.hy, lv.hz);
        __syncthreads();
      }
    }
  }
}

// clear_zero(coarse) + homogeneous ghost fill == zero every cell of the shell and interior;
// then the residual of f restricted into b of c
template <typename T>
__device__ __noinline__ void tail_restrict(const TailLevel<T> &f, const TailLevel<T> &c, int t0, int nt) {
  const int cz = c.nz + 2, cy = c.ny + 2, cx = c.nx + 2;
  for (int q = t0; q < cx * cy * cz; q += nt) {
    const int i = q / (cy * cz) - 1, j = (q / cz) % cy - 1, k = q % cz - 1;
    c.u[(long long)i * c.xs + (long long)j * c.ys + k] = (T)0;
  }
  for (int q = t0; q < c.nx * c.ny * c.nz; q += nt) {
    const int ic = q / (c.ny * c.nz), jc = (q / c.nz) % c.ny, kc = q % c.nz;
    const long long ri = (long long)(2 * ic) * f.xs + (long long)(2 * jc) * f.ys + 2 * kc;
    T r[8];
    const long long off[8] = {0, 1, f.ys, 1 + f.ys, f.xs, 1 + f.xs, f.ys + f.xs, 1 + f.ys + f.xs};
#pragma unroll
    for (int n = 0; n < 8; n++) r[n] = residual_at<T>(f.u, f.b, ri + off[n], f.xs, f.ys, f.res);
    c.b[(long long)ic * c.xs + (long long)jc * c.ys + kc] =
        (T)0.125 * (r[0] + r[1] + r[2] + r[3] + r[4] + r[5] + r[6] + r[7]);
  }
  __syncthreads();
}

// The coarsest level: the host routine's arithmetic by the CTA (block-wide), or the device
// colour sweeps.
template <typename T>
__device__ __noinline__ void tail_coarsest(const TailLevel<T> &cl, const TailParams<T> &P, int t0, int nt) {
  if (P.host_coarse) {
    coarse_relax_block<T>(cl.u, cl.b, cl.xs, cl.ys, cl.nx, cl.ny, cl.nz, P.coarse_iters, P.coarse_order, P.cc,
                          cl.bc, cl.hx, cl.hy, cl.hz);
  } else {
    tail_relax<T>(cl, P.coarse_iters, P.coarse_order, t0, nt);
  }
  __syncthreads();
}

// prolongation of c into f with f's ghosts
template <typename T>
__device__ __noinline__ void tail_prolong(const TailLevel<T> &f, const TailLevel<T> &c, int t0, int nt) {
  GhostEmit<T> ge{f.u, f.xs, f.ys, f.nx, f.ny, f.nz, f.bc, f.hx, f.hy, f.hz};
  for (int q = t0; q < c.nx * c.ny * c.nz; q += nt) {
    const int ic = q / (c.ny * c.nz), jc = (q / c.nz) % c.ny, kc = q % c.nz;
    const long long tc = (long long)ic * c.xs + (long long)jc * c.ys + kc;
    const long long fi = (long long)(2 * ic + 1) * f.xs + (long long)(2 * jc + 1) * f.ys + (2 * kc + 1);
    if (f.emit_ok)
      prolong_cell<T, true, long long>(c.u, tc, c.xs, c.ys, f.u, fi, f.xs, f.ys, ic, jc, kc, &ge);
    else
      prolong_cell<T, false, long long>(c.u, tc, c.xs, c.ys, f.u, fi, f.xs, f.ys, ic, jc, kc, nullptr);
  }
  __syncthreads();
  if (!f.emit_ok) {
    level1_fill_block<T>(f.u, f.xs, f.ys, f.nx, f.ny, f.nz, f.bc, f.hx, f.hy, f.hz);
    __syncthreads();
  }
}

// The tail schedule on level descriptors lv[0..nlev-1] (lv[0] = level s), held in shared
// memory.  Works on global memory or on a shared-memory copy; the arithmetic is the same.
template <typename T>
__device__ void tail_body(const TailLevel<T> *lv, const TailParams<T> &P, int t0, int nt) {
  const int L = P.nlev;
  for (int l = 0; l < L - 1; l++) {
    tail_relax<T>(lv[l], P.nu1, 0, t0, nt);
    tail_restrict<T>(lv[l], lv[l + 1], t0, nt);
  }
  tail_coarsest<T>(lv[L - 1], P, t0, nt);
  for (int l = L - 2; l >= 0; l--) {
    tail_prolong<T>(lv[l], lv[l + 1], t0, nt);
    if (P.first_level + l > 0) tail_relax<T>(lv[l], P.nu2, P.post_order, t0, nt);
  }
}

// Member of this CTA, or -1 when its state does not select it (single grid: member 0).
__device__ __forceinline__ int batch_member(const BatchSel &sel, int m) {
  if (!sel.state) return 0;
  return sel.state[m] == sel.want ? m : -1;
}

template <typename T>
__global__ void __launch_bounds__(1024) k_coarse_tail(const __grid_constant__ TailParams<T> P,
                                                      const __grid_constant__ TailBatch tb) {
  pdl_entry();
  __shared__ TailLevel<T> lv[kMaxTailLevels];
  const int m = batch_member(tb.sel, blockIdx.x);
  if (m < 0) return;
  if (threadIdx.x < P.nlev) {
    TailLevel<T> d = P.lv[threadIdx.x];
    d.u += m * tb.ms[threadIdx.x];
    d.b += m * tb.ms[threadIdx.x];
    lv[threadIdx.x] = d;
  }
  __syncthreads();
  tail_body<T>(lv, P, threadIdx.x, blockDim.x);
}

// Shared-memory variant: every tail level's u and b (interior + ghost shell, compact strides)
// is staged in dynamic shared memory, the schedule runs there, and u (shell included) and the
// interior of b are written back.  Only level s is read: the lower levels are zeroed /
// restricted inside the schedule before they are used.
template <typename T>
__global__ void __launch_bounds__(512) k_coarse_tail_smem(const __grid_constant__ TailParams<T> P,
                                                           const __grid_constant__ TailBatch tb) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ TailLevel<T> lv[kMaxTailLevels];
  __shared__ TailLevel<T> gl[kMaxTailLevels];  // this member's levels in global memory
  const int m = batch_member(tb.sel, blockIdx.x);
  if (m < 0) return;
  const int L = P.nlev;
  if (threadIdx.x < L) {
    TailLevel<T> d = P.lv[threadIdx.x];
    d.u += m * tb.ms[threadIdx.x];
    d.b += m * tb.ms[threadIdx.x];
    gl[threadIdx.x] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    T *cur = reinterpret_cast<T *>(smem_raw);
    for (int l = 0; l < L; l++) {
      TailLevel<T> d = gl[l];
      const long long sys = d.nz + 2, sxs = (long long)(d.ny + 2) * (d.nz + 2);
      const long long cells = (long long)(d.nx + 2) * sxs;
      d.xs = sxs;
      d.ys = sys;
      d.u = cur + sxs + sys + 1;
      cur += cells;
      d.b = cur + sxs + sys + 1;
      cur += cells;
      lv[l] = d;
    }
  }
  __syncthreads();
  const int nt = blockDim.x;
  {  // stage level s
    const TailLevel<T> &g = gl[0];
    const TailLevel<T> &sh = lv[0];
    const int cz = g.nz + 2, cy = g.ny + 2, cx = g.nx + 2;
    for (int q = threadIdx.x; q < cx * cy * cz; q += nt) {
      const int i = q / (cy * cz) - 1, j = (q / cz) % cy - 1, k = q % cz - 1;
      sh.u[(long long)i * sh.xs + (long long)j * sh.ys + k] = g.u[(long long)i * g.xs + (long long)j * g.ys + k];
      sh.b[(long long)i * sh.xs + (long long)j * sh.ys + k] = g.b[(long long)i * g.xs + (long long)j * g.ys + k];
    }
  }
  __syncthreads();
  tail_body<T>(lv, P, threadIdx.x, nt);
  __syncthreads();
  for (int l = 0; l < L; l++) {  // write back: u with its ghost shell, b interior below level s
    const TailLevel<T> &g = gl[l];
    const TailLevel<T> &sh = lv[l];
    const int cz = g.nz + 2, cy = g.ny + 2, cx = g.nx + 2;
    for (int q = threadIdx.x; q < cx * cy * cz; q += nt) {
      const int i = q / (cy * cz) - 1, j = (q / cz) % cy - 1, k = q % cz - 1;
      const long long gi = (long long)i * g.xs + (long long)j * g.ys + k;
      const long long si = (long long)i * sh.xs + (long long)j * sh.ys + k;
      g.u[gi] = sh.u[si];
      if (l > 0 && i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz) g.b[gi] = sh.b[si];
    }
  }
}

template <typename T>
size_t tail_smem_bytes(const TailParams<T> &P) {
  size_t cells = 0;
  for (int l = 0; l < P.nlev; l++) cells += 2 * (size_t)(P.lv[l].nx + 2) * (P.lv[l].ny + 2) * (P.lv[l].nz + 2);
  return cells * sizeof(T);
}

template <typename T>
ocu_status launch_coarse_tail_batch(const TailParams<T> &P, const TailBatch &tb, int members, cudaStream_t s) {
  const size_t bytes = tail_smem_bytes<T>(P);
  constexpr size_t kMaxSmem = 200 * 1024;
  if (bytes <= kMaxSmem) {
    static std::atomic<unsigned long long> attr_set{0};  // one bit per device, per instance
    int dev = 0;
    OCU_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_set.load() & bit)) {
      OCU_TRY(check_cuda(cudaFuncSetAttribute(k_coarse_tail_smem<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kMaxSmem),
                         "cudaFuncSetAttribute(k_coarse_tail_smem)"));
      attr_set.fetch_or(bit);
    }
    // one warp-multiple of threads per ~2 cells of the largest level: small tails take 256
    const long long top = (long long)P.lv[0].nx * P.lv[0].ny * P.lv[0].nz;
    launch_pdl(k_coarse_tail_smem<T>, members, top <= 512 ? 256 : 512, bytes, s, P, tb);
    return check_launch("k_coarse_tail_smem");
  }
  launch_pdl(k_coarse_tail<T>, members, 1024, 0, s, P, tb);
  return check_launch("k_coarse_tail");
}

template <typename T>
ocu_status launch_coarse_tail(const TailParams<T> &P, cudaStream_t s) {
  TailBatch tb;
  std::memset(&tb, 0, sizeof(tb));
  return launch_coarse_tail_batch<T>(P, tb, 1, s);
}

// ------------------------------------------------------------------------------------------
// Ensemble (batched) kernels: the same cell arithmetic as the single-grid kernels above, over
// `members` congruent grids laid out at base + m * ms.  blockIdx.z carries (member, z block);
// members whose state differs from sel.want return at once.  Each member's result is
// bit-identical to the single-grid kernel applied to that member alone.
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 6) k_relax_color_emit_b(T *__restrict__ u, const T *__restrict__ b, long long xs,
                                                            long long ys, int nx, int ny, int nz, int color,
                                                            RelaxCoefD<T> c, const T *__restrict__ diag,
                                                            const __grid_constant__ GhostEmit<T> ge, BatchSel sel,
                                                            long long ms, int zb) {
  pdl_entry();
  const int m = batch_member(sel, blockIdx.z / zb);
  if (m < 0) return;
  const int bz = blockIdx.z % zb;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = bz * blockDim.z + threadIdx.z;
  const bool edge_block = color_edge_block(blockIdx.x, blockIdx.y, bz, nx, ny, nz);
  if (i >= nx || j >= ny || t >= nz / 2) return;
  u += m * ms;
  b += m * ms;
  GhostEmit<T> g = ge;
  g.p = u;
  color_cell<T, int, true>(u, b, (int)xs, (int)ys, i, j, 2 * t + ((i + j + color) & 1), nx, ny, nz, c, diag, edge_block,
                           g);
}

template <typename T>
ocu_status launch_relax_color_emit_b(T *u, const T *b, const ocu_layout &L, const T *diag, int color,
                                     const RelaxParams &p, double hx, double hy, double hz, const BatchSel &sel,
                                     long long ms, int members, const int block[3], cudaStream_t s) {
  const RelaxCoefD<T> c = make_relax_coef_d<T>(p);
  const int half = L.nz / 2;
  if (half == 0) return OCU_OK;
  dim3 bl(block[0], block[1], block[2]);
  if ((int)bl.x > half) bl.x = half >= 16 ? 16 : (half >= 8 ? 8 : (half >= 4 ? 4 : half));
  const int zb = (L.nx + bl.z - 1) / bl.z;
  if ((long long)zb * members > 65535)
    return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ensemble - too many members of size (%d,%d,%d) in one class", L.nx, L.ny, L.nz);
  dim3 grid((half + bl.x - 1) / bl.x, (L.ny + bl.y - 1) / bl.y, (unsigned)(zb * members));
  GhostEmit<T> ge{u, L.xstride, L.ystride, L.nx, L.ny, L.nz, to_dev(p.bc), (T)hx, (T)hy, (T)hz};
  launch_pdl(k_relax_color_emit_b<T>, grid, bl, 0, s, u, b, L.xstride, L.ystride, L.nx, L.ny, L.nz, color, c, diag, ge,
             sel, ms, zb);
  return check_launch("k_relax_color_emit_b");
}

template <typename T>
__global__ void __launch_bounds__(256, 3) k_prolong_emit_b(const T *__restrict__ uc, long long cx, long long cy,
                                                           int cnx, int cny, int cnz, T *__restrict__ uf,
                                                           long long fxs, long long fys,
                                                           const __grid_constant__ GhostEmit<T> ge, BatchSel sel,
                                                           long long cms, long long fms) {
  pdl_entry();
  const int m = batch_member(sel, blockIdx.z / cnx);
  if (m < 0) return;
  const int ic = blockIdx.z % cnx;
  const int kc = blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  if (kc >= cnz || jc >= cny) return;
  uc += m * cms;
  uf += m * fms;
  const int tc = ic * (int)cx + jc * (int)cy + kc;
  const int f = (2 * ic + 1) * (int)fxs + (2 * jc + 1) * (int)fys + (2 * kc + 1);
  if (ic == 0 || ic == cnx - 1 || jc == 0 || jc == cny - 1 || kc == 0 || kc == cnz - 1) {
    GhostEmit<T> g = ge;
    g.p = uf;
    prolong_cell<T, true, int>(uc, tc, (int)cx, (int)cy, uf, f, (int)fxs, (int)fys, ic, jc, kc, &g);
  } else {
    prolong_cell<T, false, int>(uc, tc, (int)cx, (int)cy, uf, f, (int)fxs, (int)fys, ic, jc, kc, nullptr);
  }
}

template <typename T>
ocu_status launch_prolong_emit_b(const T *uc, const ocu_layout &Lc, T *uf, const ocu_layout &Lf,
                                 const ocu_bc_set &bc_fine, double hx, double hy, double hz, const BatchSel &sel,
                                 long long cms, long long fms, int members, cudaStream_t s) {
  dim3 block(Lc.nz >= 32 ? 32 : 16, 8);
  if ((long long)Lc.nx * members > 65535)
    return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ensemble - too many members of one size in one class");
  dim3 grid((Lc.nz + block.x - 1) / block.x, (Lc.ny + block.y - 1) / block.y, (unsigned)(Lc.nx * members));
  GhostEmit<T> ge{uf, Lf.xstride, Lf.ystride, Lf.nx, Lf.ny, Lf.nz, to_dev(bc_fine), (T)hx, (T)hy, (T)hz};
  launch_pdl(k_prolong_emit_b<T>, grid, block, 0, s, uc, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, uf, Lf.xstride,
             Lf.ystride, ge, sel, cms, fms);
  return check_launch("k_prolong_emit_b");
}

// Residual + restriction (+ level-0 norm partials) per member; rows of member m at
// rows + m * nrows (nrows = fine nx * ny).
template <typename T, bool NORM>
__global__ void __launch_bounds__(256) k_residual_restrict_b(const T *__restrict__ u, const T *__restrict__ b,
                                                             long long xs, long long ys, int nx, int ny, int nz,
                                                             ResCoefT<T> c, T *__restrict__ bc_, long long bxs,
                                                             long long bys, int cnx, int cny, int cnz,
                                                             T *__restrict__ rows2, BatchSel sel, long long fms,
                                                             long long cms) {
  pdl_entry();
  const int m = batch_member(sel, blockIdx.z / cnx);
  if (m < 0) return;
  const int ic = blockIdx.z % cnx;
  const int lane = threadIdx.x;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  if (jc >= cny) return;
  u += m * fms;
  b += m * fms;
  bc_ += m * cms;
  T acc2[4] = {0, 0, 0, 0}, accinf[4] = {0, 0, 0, 0};
  const long long frow = (long long)(2 * ic) * xs + (long long)(2 * jc) * ys;
  for (int cbase = 0; cbase < cnz; cbase += 32) {
    const int kc = cbase + lane;
    T r[8];
    if (kc < cnz) {
      const long long ri = frow + 2 * kc;
      r[0] = residual_at<T>(u, b, ri, xs, ys, c);
      r[1] = residual_at<T>(u, b, ri + 1, xs, ys, c);
      r[2] = residual_at<T>(u, b, ri + ys, xs, ys, c);
      r[3] = residual_at<T>(u, b, ri + 1 + ys, xs, ys, c);
      r[4] = residual_at<T>(u, b, ri + xs, xs, ys, c);
      r[5] = residual_at<T>(u, b, ri + 1 + xs, xs, ys, c);
      r[6] = residual_at<T>(u, b, ri + ys + xs, xs, ys, c);
      r[7] = residual_at<T>(u, b, ri + 1 + ys + xs, xs, ys, c);
      bc_[(long long)ic * bxs + (long long)jc * bys + kc] =
          (T)0.125 * (r[0] + r[1] + r[2] + r[3] + r[4] + r[5] + r[6] + r[7]);
    } else {
#pragma unroll
      for (int q = 0; q < 8; q++) r[q] = 0;
    }
    if (NORM) {
#pragma unroll
      for (int q = 0; q < 4; q++)
        fold_chunk<T>(r[2 * q], r[2 * q + 1], 2 * cbase, nz, lane, acc2[q], accinf[q], true, false);
    }
  }
  if (NORM) {
    T *rows = rows2 + (long long)m * nx * ny;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * ic + (q >> 1), j = 2 * jc + (q & 1);
      const T v = warp_tree<T>(acc2[q], false);
      if (lane == 0) rows[(long long)i * ny + j] = v;
    }
  }
}

template <typename T>
ocu_status launch_residual_restrict_b(const T *u, const T *b, const ocu_layout &Lf, T *bc_, const ocu_layout &Lc,
                                      double h, double fx, double fy, double fz, T *rows2, const BatchSel &sel,
                                      long long fms, long long cms, int members, cudaStream_t s) {
  if ((long long)Lc.nx * members > 65535)
    return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ensemble - too many members of one size in one class");
  dim3 block(32, 8), grid(1, (Lc.ny + 7) / 8, (unsigned)(Lc.nx * members));
  const ResCoefT<T> c = res_coef<T>(h, fx, fy, fz);
  if (rows2)
    launch_pdl(k_residual_restrict_b<T, true>, grid, block, 0, s, u, b, Lf.xstride, Lf.ystride, Lf.nx, Lf.ny, Lf.nz, c,
               bc_, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, rows2, sel, fms, cms);
  else
    launch_pdl(k_residual_restrict_b<T, false>, grid, block, 0, s, u, b, Lf.xstride, Lf.ystride, Lf.nx, Lf.ny, Lf.nz, c,
               bc_, Lc.xstride, Lc.ystride, Lc.nx, Lc.ny, Lc.nz, nullptr, sel, fms, cms);
  return check_launch("k_residual_restrict_b");
}

// Residual norm partials of level 0 (no restriction), per member.
template <typename T>
__global__ void __launch_bounds__(256) k_residual_rows_b(const T *__restrict__ u, const T *__restrict__ b,
                                                         long long xs, long long ys, int nx, int ny, int nz,
                                                         ResCoefT<T> c, T *__restrict__ rows2, BatchSel sel,
                                                         long long ms) {
  pdl_entry();
  const int m = batch_member(sel, blockIdx.z / nx);
  if (m < 0) return;
  const int i = blockIdx.z % nx;
  const int lane = threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= ny) return;
  u += m * ms;
  b += m * ms;
  T acc2 = 0, accinf = 0;
  const long long row = (long long)i * xs + (long long)j * ys;
  for (int base = 0; base < nz; base += 64) {
    const int k0 = base + 2 * lane;
    T e0 = 0, e1 = 0;
    if (k0 < nz) e0 = residual_at<T>(u, b, row + k0, xs, ys, c);
    if (k0 + 1 < nz) e1 = residual_at<T>(u, b, row + k0 + 1, xs, ys, c);
    fold_chunk<T>(e0, e1, base, nz, lane, acc2, accinf, true, false);
  }
  const T v = warp_tree<T>(acc2, false);
  if (lane == 0) rows2[(long long)m * nx * ny + (long long)i * ny + j] = v;
}

template <typename T>
ocu_status launch_residual_rows_b(const T *u, const T *b, const ocu_layout &L, double h, double fx, double fy,
                                  double fz, T *rows2, const BatchSel &sel, long long ms, int members,
                                  cudaStream_t s) {
  if ((long long)L.nx * members > 65535)
    return fail(OCU_ERR_UNSUPPORTED, "[ERROR] ensemble - too many members of one size in one class");
  dim3 block(32, 8), grid(1, (L.ny + 7) / 8, (unsigned)(L.nx * members));
  launch_pdl(k_residual_rows_b<T>, grid, block, 0, s, u, b, L.xstride, L.ystride, L.nx, L.ny, L.nz,
             res_coef<T>(h, fx, fy, fz), rows2, sel, ms);
  return check_launch("k_residual_rows_b");
}

// Per-member fold of the row sums, one CTA per member, in exactly k_fold_rows' order: 256-row
// blocks folded by a 256-wide tree into partials, then the partials folded 256 at a time.
template <typename T>
__global__ void __launch_bounds__(256) k_fold_rows_b(const T *__restrict__ rows, long long nrows, T *partial,
                                                     long long pstride, double *sums, BatchSel sel) {
  pdl_entry();
  __shared__ T sh[256];
  const int m = batch_member(sel, blockIdx.x);
  if (m < 0) return;
  rows += (long long)m * nrows;
  T *part = partial + (long long)m * pstride;
  const long long nb = (nrows + 255) / 256;
  for (long long bb = 0; bb < nb; bb++) {
    const long long idx = bb * 256 + threadIdx.x;
    sh[threadIdx.x] = idx < nrows ? rows[idx] : (T)0;
    __syncthreads();
    for (int stride = 128; stride > 0; stride >>= 1) {
      if (threadIdx.x < stride) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + stride];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[bb] = sh[0];
    __syncthreads();
  }
  long long count = nb;
  while (count > 1) {
    const long long nb2 = (count + 255) / 256;
    for (long long bb = 0; bb < nb2; bb++) {
      const long long q = bb * 256 + threadIdx.x;
      sh[threadIdx.x] = q < count ? part[q] : (T)0;
      __syncthreads();
      for (int stride = 128; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + stride];
        __syncthreads();
      }
      if (threadIdx.x == 0) part[bb] = sh[0];
      __syncthreads();
    }
    count = nb2;
  }
  if (threadIdx.x == 0) sums[m] = (double)part[0];
}

template <typename T>
ocu_status launch_fold_rows_b(const T *rows, long long nrows, T *partial, long long pstride, double *sums,
                              const BatchSel &sel, int members, cudaStream_t s) {
  launch_pdl(k_fold_rows_b<T>, members, 256, 0, s, rows, nrows, partial, pstride, sums, sel);
  return check_launch("k_fold_rows_b");
}

// Level-1 ghost fill of each selected member (one CTA per member); with `retire` the member's
// state is set to 0 afterwards (members that converged this cycle get their final fill).
template <typename T>
__global__ void __launch_bounds__(512) k_bc_fill_b(T *u, long long xs, long long ys, int nx, int ny, int nz,
                                                   const __grid_constant__ BCDev bc, T hx, T hy, T hz, BatchSel sel,
                                                   long long ms, int *state, int retire) {
  pdl_entry();
  const int m = batch_member(sel, blockIdx.x);
  if (m < 0) return;
  level1_fill_block<T>(u + m * ms, xs, ys, nx, ny, nz, bc, hx, hy, hz);
  if (retire) {
    __syncthreads();  // every thread has read state[m] before it changes
    if (threadIdx.x == 0) state[m] = 0;
  }
}

template <typename T>
ocu_status launch_bc_fill_b(T *u, const ocu_layout &L, const ocu_bc_set &bc, double hx, double hy, double hz,
                            const BatchSel &sel, long long ms, int members, int *state, bool retire,
                            cudaStream_t s) {
  launch_pdl(k_bc_fill_b<T>, members, 512, 0, s, u, L.xstride, L.ystride, L.nx, L.ny, L.nz, to_dev(bc), (T)hx, (T)hy,
             (T)hz, sel, ms, state, retire ? 1 : 0);
  return check_launch("k_bc_fill_b");
}

// Convergence decision of every active member, as the host driver makes it: l2 = sqrt(sum / N)
// in T, converged when l2 < tol (sol_mgpressure3d.cpp:186-236).  initial: the check before any
// cycle (converged members are done: state 0); otherwise a counted cycle (converged: state 2,
// so the final ghost fill runs).  Writes the number of members still active to *active.
template <typename T>
__global__ void __launch_bounds__(1024) k_converge_b(const double *sums, long long ncell, const double *tol,
                                                     int *state, int *vcycles, double *last_l2, int *active,
                                                     int members, int initial) {
  pdl_entry();
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int m = threadIdx.x; m < members; m += blockDim.x) {
    if (state[m] != 1) continue;
    T rn = (T)sums[m];
    rn /= (T)ncell;
    const double l2 = (double)sqrt(rn);
    last_l2[m] = l2;
    if (!initial) vcycles[m] += 1;
    if (l2 < tol[m]) {
      state[m] = initial ? 0 : 2;
    } else {
      mine++;
    }
  }
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) *active = cnt;
}

template <typename T>
ocu_status launch_converge_b(const double *sums, long long ncell, const double *tol, int *state, int *vcycles,
                             double *last_l2, int *active, int members, bool initial, cudaStream_t s) {
  launch_pdl(k_converge_b<T>, 1, 1024, 0, s, sums, ncell, tol, state, vcycles, last_l2, active, members, initial ? 1 : 0);
  return check_launch("k_converge_b");
}

#define INST_B(T)                                                                                              \
  template ocu_status launch_relax_color_emit_b<T>(T *, const T *, const ocu_layout &, const T *, int,         \
                                                   const RelaxParams &, double, double, double,                \
                                                   const BatchSel &, long long, int, const int[3],             \
                                                   cudaStream_t);                                              \
  template ocu_status launch_prolong_emit_b<T>(const T *, const ocu_layout &, T *, const ocu_layout &,         \
                                               const ocu_bc_set &, double, double, double, const BatchSel &,   \
                                               long long, long long, int, cudaStream_t);                       \
  template ocu_status launch_residual_restrict_b<T>(const T *, const T *, const ocu_layout &, T *,              \
                                                    const ocu_layout &, double, double, double, double, T *,    \
                                                    const BatchSel &, long long, long long, int, cudaStream_t); \
  template ocu_status launch_residual_rows_b<T>(const T *, const T *, const ocu_layout &, double, double,       \
                                                double, double, T *, const BatchSel &, long long, int,          \
                                                cudaStream_t);                                                 \
  template ocu_status launch_fold_rows_b<T>(const T *, long long, T *, long long, double *, const BatchSel &,    \
                                            int, cudaStream_t);                                                \
  template ocu_status launch_bc_fill_b<T>(T *, const ocu_layout &, const ocu_bc_set &, double, double, double,  \
                                          const BatchSel &, long long, int, int *, bool, cudaStream_t);        \
  template ocu_status launch_converge_b<T>(const double *, long long, const double *, int *, int *, double *,    \
                                           int *, int, bool, cudaStream_t);
INST_B(float)
INST_B(double)
#undef INST_B

#define INST(T)                                                                                                \
  template ocu_status launch_relax_color_emit<T>(T *, const T *, const ocu_layout &, const T *, int,           \
                                                 const RelaxParams &, double, double, double, cudaStream_t);  \
  template ocu_status launch_prolong_emit<T>(const T *, const ocu_layout &, T *, const ocu_layout &,           \
                                             const ocu_bc_set &, double, double, double, cudaStream_t);       \
  template ocu_status launch_residual_rows<T>(const T *, const T *, T *, float *, const ocu_layout &, double,   \
                                              double, double, double, T *, T *, cudaStream_t);                 \
  template ocu_status launch_residual_restrict<T>(const T *, const T *, const ocu_layout &, T *,                \
                                                  const ocu_layout &, double, double, double, double, T *, T *, \
                                                  cudaStream_t, T *, long long);                               \
  template ocu_status launch_fold_rows<T>(const T *, long long, bool, void *, double *, cudaStream_t);          \
  template ocu_status launch_coarse_tail<T>(const TailParams<T> &, cudaStream_t);                               \
  template ocu_status launch_coarse_tail_batch<T>(const TailParams<T> &, const TailBatch &, int, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace ocub
