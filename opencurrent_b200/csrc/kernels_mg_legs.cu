// One launch per V-cycle leg on the small levels.
//
// Below a few ten thousand cells a level's kernels are latency-bound: each colour sweep,
// residual + restriction, clear and prolongation is a dependent launch of a few microseconds
// that does almost no work.  Here the down-leg of a level (nu1 red-black iterations, the residual,
// its restriction into the coarser level's b, and the coarser level's clear) and its up-leg
// (prolongation + correction, nu2 iterations) are each ONE launch.  Every CTA owns a box of the
// level (8 x 8 x 16 cells), stages the box plus a halo of H cells in shared memory (H = 2*nu + 1
// for the down-leg, 2*nu for the up-leg) and runs all the colour passes there; pass p is valid
// on the box grown by H-1-p, so the halo is relaxed redundantly instead of exchanged.  Periodic
// axes are staged by wrapping (the periodic ghost of a cell always equals the cell it copies),
// Dirichlet/Neumann face ghosts are recomputed in shared memory after every pass with the ghost
// rule of the separate fill.  The result is written out of place (the level's second u buffer
// and back), because other CTAs may still be staging the cells a CTA owns.  The arithmetic per
// cell is that of the per-operation kernels: relax_value, residual_at and the prolongation
// child sums in the same operand order, so the results are bit-identical.
#include "bc_device.cuh"
#include "ghost_emit.cuh"
#include "mg_fused.h"
#include "mg_solver.h"
#include "ocu_internal.h"
#include "relax_math.cuh"

#include <atomic>

namespace ocub {

namespace {

constexpr int kLegThreads = 1024;

// box of a CTA along x, y, z
__host__ __device__ constexpr int leg_tile(int a) { return a == 2 ? 16 : 8; }
__host__ __device__ constexpr int leg_region(int a) { return leg_tile(a) + 2 * kLegMaxHalo; }
__host__ __device__ constexpr int leg_coarse_region(int a) { return leg_region(a) / 2 + 3; }

__device__ __forceinline__ int wrapc(int c, int n) {
  c %= n;
  return c < 0 ? c + n : c;
}

// Per-CTA geometry: the box [b0, b1), the staged region [r0, r1) (logical coordinates: periodic
// axes unwrapped, others clipped to the ghost layer [-1, n]) and its shared-memory strides.
struct LegGeom {
  int b0[3], b1[3], r0[3], r1[3];
  int sx, sy;  // region strides (z contiguous)
};

template <typename T>
__device__ __forceinline__ LegGeom leg_geom(const LegLevel<T> &P, int halo) {
  LegGeom g;
  const int blk[3] = {(int)blockIdx.z, (int)blockIdx.y, (int)blockIdx.x};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    g.b0[a] = blk[a] * leg_tile(a);
    g.b1[a] = min(g.b0[a] + leg_tile(a), P.n[a]);
    g.r0[a] = g.b0[a] - halo;
    g.r1[a] = g.b1[a] + halo;
    if (!P.per[a]) {
      g.r0[a] = max(g.r0[a], -1);
      g.r1[a] = min(g.r1[a], P.n[a] + 1);
    }
  }
  g.sy = g.r1[2] - g.r0[2];
  g.sx = (g.r1[1] - g.r0[1]) * g.sy;
  return g;
}

// Global element offset of logical cell (i, j, k) (periodic axes wrapped).
template <typename T>
__device__ __forceinline__ long long leg_phys(const LegLevel<T> &P, int i, int j, int k) {
  if (P.per[0]) i = wrapc(i, P.n[0]);
  if (P.per[1]) j = wrapc(j, P.n[1]);
  if (P.per[2]) k = wrapc(k, P.n[2]);
  return (long long)i * P.xs + (long long)j * P.ys + k;
}

// Stage u (region) and b (its interior part) in shared memory.
template <typename T>
__device__ void leg_stage(const LegLevel<T> &P, const LegGeom &g, const T *__restrict__ u, T *us, T *bs) {
  const int ny = g.r1[1] - g.r0[1], nz = g.sy;
  const int cells = (g.r1[0] - g.r0[0]) * ny * nz;
  for (int q = threadIdx.x; q < cells; q += blockDim.x) {
    const int a = q / (ny * nz), rem = q - a * (ny * nz), b = rem / nz, c = rem - b * nz;
    const int i = g.r0[0] + a, j = g.r0[1] + b, k = g.r0[2] + c;
    const long long id = leg_phys(P, i, j, k);
    us[q] = u[id];
    const bool inside = (P.per[0] || (i >= 0 && i < P.n[0])) && (P.per[1] || (j >= 0 && j < P.n[1])) &&
                        (P.per[2] || (k >= 0 && k < P.n[2]));
    bs[q] = inside ? P.b[id] : (T)0;
  }
}

// Recompute the Dirichlet/Neumann face ghosts of the region from their source cells (the
// separate fill's x, y or z rule; edge and corner ghosts are never read by 7-point stencils).
template <typename T>
__device__ void leg_face_ghosts(const LegLevel<T> &P, const LegGeom &g, T *us, const GhostEmit<T> &ge) {
  const int str[3] = {g.sx, g.sy, 1};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (P.per[a]) continue;
    const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;  // the other two axes
    // their interior (or periodic) extent inside the region
    const int lob = P.per[b] ? g.r0[b] : max(g.r0[b], 0), hib = P.per[b] ? g.r1[b] : min(g.r1[b], P.n[b]);
    const int loc = P.per[c] ? g.r0[c] : max(g.r0[c], 0), hic = P.per[c] ? g.r1[c] : min(g.r1[c], P.n[c]);
    const int nb = hib - lob, nc = hic - loc;
    if (nb <= 0 || nc <= 0) continue;
#pragma unroll
    for (int side = 0; side < 2; side++) {
      const int gc = side ? P.n[a] : -1;  // ghost coordinate
      if (gc < g.r0[a] || gc >= g.r1[a]) continue;
      const int sc = side ? P.n[a] - 1 : 0;  // its source
      if (sc < g.r0[a] || sc >= g.r1[a]) continue;
      for (int q = threadIdx.x; q < nb * nc; q += blockDim.x) {
        const int xb = lob + q / nc, xc = loc + q % nc;
        const int off = (xb - g.r0[b]) * str[b] + (xc - g.r0[c]) * str[c];
        const T src = us[off + (sc - g.r0[a]) * str[a]];
        T v;
        if (a == 0) v = side ? ge.template rule<FX_POS>(src, P.h[0]) : ge.template rule<FX_NEG>(src, P.h[0]);
        else if (a == 1) v = side ? ge.template rule<FY_POS>(src, P.h[1]) : ge.template rule<FY_NEG>(src, P.h[1]);
        else v = side ? ge.template rule<FZ_POS>(src, P.h[2]) : ge.template rule<FZ_NEG>(src, P.h[2]);
        us[off + (gc - g.r0[a]) * str[a]] = v;
      }
    }
  }
}

// `passes` colour passes (the colour order of one relax(level, passes/2, order) call), pass p over
// the cells of its colour in the box grown by grow0 - p, each followed by the face-ghost refresh.
template <typename T>
__device__ void leg_relax(const LegLevel<T> &P, const LegGeom &g, T *us, const T *bs, int passes, int order,
                          int grow0, const GhostEmit<T> &ge) {
  for (int p = 0; p < passes; p++) {
    const int rb = p & 1;
    const int color = order == RO_BLACK_RED ? !rb : rb;
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      lo[a] = g.b0[a] - (grow0 - p);
      hi[a] = g.b1[a] + (grow0 - p);
      if (!P.per[a]) {
        lo[a] = max(lo[a], 0);
        hi[a] = min(hi[a], P.n[a]);
      }
    }
    const int vy = hi[1] - lo[1], vz = hi[2] - lo[2], hz = (vz + 1) / 2;
    const int work = (hi[0] - lo[0]) * vy * hz;
    for (int q = threadIdx.x; q < work; q += blockDim.x) {
      const int row = q / hz, s = q - row * hz;
      const int i = lo[0] + row / vy, j = lo[1] + row % vy;
      const int k = lo[2] + ((color - i - j - lo[2]) & 1) + 2 * s;  // (i + j + k) has the colour's parity
      if (k >= hi[2]) continue;
      const int r = (i - g.r0[0]) * g.sx + (j - g.r0[1]) * g.sy + (k - g.r0[2]);
      const int iw = P.per[0] ? wrapc(i, P.n[0]) : i, jw = P.per[1] ? wrapc(j, P.n[1]) : j,
                kw = P.per[2] ? wrapc(k, P.n[2]) : k;
      us[r] = relax_value<T>(us[r], bs[r], us[r - 1], us[r + 1], us[r - g.sy], us[r + g.sy], us[r - g.sx],
                             us[r + g.sx], iw, jw, kw, P.n[0], P.n[1], P.n[2], P.rc, nullptr);
    }
    __syncthreads();
    leg_face_ghosts<T>(P, g, us, ge);
    __syncthreads();
  }
}

// The box back to global memory (out of place) with every ghost its boundary cells source.
template <typename T>
__device__ void leg_write_box(const LegLevel<T> &P, const LegGeom &g, const T *us, const GhostEmit<T> &ge) {
  const int ny = g.b1[1] - g.b0[1], nz = g.b1[2] - g.b0[2];
  const int cells = (g.b1[0] - g.b0[0]) * ny * nz;
  for (int q = threadIdx.x; q < cells; q += blockDim.x) {
    const int a = q / (ny * nz), rem = q - a * (ny * nz), b = rem / nz;
    const int i = g.b0[0] + a, j = g.b0[1] + b, k = g.b0[2] + (rem - b * nz);
    const T v = us[(i - g.r0[0]) * g.sx + (j - g.r0[1]) * g.sy + (k - g.r0[2])];
    P.u_out[(long long)i * P.xs + (long long)j * P.ys + k] = v;
    ge.emit(i, j, k, v);
  }
}

template <typename T>
__device__ __forceinline__ GhostEmit<T> leg_emitter(const LegLevel<T> &P) {
  return GhostEmit<T>{P.u_out, P.xs, P.ys, P.n[0], P.n[1], P.n[2], P.bc, P.h[0], P.h[1], P.h[2]};
}

}  // namespace

// Down-leg: relax(level, nu1, RO_RED_BLACK), clear(level+1), restriction of the residual.
template <typename T>
__global__ void __launch_bounds__(kLegThreads) k_leg_down(const __grid_constant__ LegLevel<T> P) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char leg_smem[];
  T *us = reinterpret_cast<T *>(leg_smem);
  T *bs = us + leg_region(0) * leg_region(1) * leg_region(2);
  {  // clear the coarser level (every element, as the memset it replaces): nothing here reads it
    const long long nthreads = (long long)gridDim.x * gridDim.y * gridDim.z * blockDim.x;
    const long long tid =
        ((long long)(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x;
    for (long long q = tid; q < P.c_alloc; q += nthreads) P.cu_base[q] = (T)0;
  }
  const int halo = P.passes + 1;
  const LegGeom g = leg_geom<T>(P, halo);
  const GhostEmit<T> ge = leg_emitter<T>(P);
  leg_stage<T>(P, g, P.u_in, us, bs);
  __syncthreads();
  leg_relax<T>(P, g, us, bs, P.passes, RO_RED_BLACK, halo - 1, ge);
  // residual of the 8 children of each coarse cell of the box, restricted in the order of the
  // per-operation kernels
  const int cnx = (g.b1[0] - g.b0[0]) / 2, cny = (g.b1[1] - g.b0[1]) / 2, cnz = (g.b1[2] - g.b0[2]) / 2;
  for (int q = threadIdx.x; q < cnx * cny * cnz; q += blockDim.x) {
    const int a = q / (cny * cnz), rem = q - a * (cny * cnz), b = rem / cnz, c = rem - b * cnz;
    const int ic = g.b0[0] / 2 + a, jc = g.b0[1] / 2 + b, kc = g.b0[2] / 2 + c;
    const long long ri = (long long)(2 * ic - g.r0[0]) * g.sx + (long long)(2 * jc - g.r0[1]) * g.sy + (2 * kc - g.r0[2]);
    const long long sx = g.sx, sy = g.sy;
    const T r0 = residual_at<T>(us, bs, ri, sx, sy, P.res);
    const T r1 = residual_at<T>(us, bs, ri + 1, sx, sy, P.res);
    const T r2 = residual_at<T>(us, bs, ri + sy, sx, sy, P.res);
    const T r3 = residual_at<T>(us, bs, ri + 1 + sy, sx, sy, P.res);
    const T r4 = residual_at<T>(us, bs, ri + sx, sx, sy, P.res);
    const T r5 = residual_at<T>(us, bs, ri + 1 + sx, sx, sy, P.res);
    const T r6 = residual_at<T>(us, bs, ri + sy + sx, sx, sy, P.res);
    const T r7 = residual_at<T>(us, bs, ri + 1 + sy + sx, sx, sy, P.res);
    P.cb[(long long)ic * P.cxs + (long long)jc * P.cys + kc] = (T)0.125 * (r0 + r1 + r2 + r3 + r4 + r5 + r6 + r7);
  }
  leg_write_box<T>(P, g, us, ge);
}

// Up-leg: prolong(level+1, level) (correction + ghosts), relax(level, nu2, order).
template <typename T>
__global__ void __launch_bounds__(kLegThreads) k_leg_up(const __grid_constant__ LegLevel<T> P) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char leg_smem[];
  T *us = reinterpret_cast<T *>(leg_smem);
  T *bs = us + leg_region(0) * leg_region(1) * leg_region(2);
  T *cs = bs + leg_region(0) * leg_region(1) * leg_region(2);
  const int halo = P.passes;
  const LegGeom g = leg_geom<T>(P, halo);
  const GhostEmit<T> ge = leg_emitter<T>(P);
  leg_stage<T>(P, g, P.u_in, us, bs);
  // coarse cells around the parents of the region (periodic axes wrapped, others clipped to the
  // coarse ghost layer)
  int c0[3], c1[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    c0[a] = (g.r0[a] >> 1) - 1;
    c1[a] = ((g.r1[a] - 1) >> 1) + 2;
    if (!P.per[a]) {
      c0[a] = max(c0[a], -1);
      c1[a] = min(c1[a], P.cn[a] + 1);
    }
  }
  const int csy = c1[2] - c0[2], csx = (c1[1] - c0[1]) * csy;
  {
    const int ny = c1[1] - c0[1], nz = csy, cells = (c1[0] - c0[0]) * ny * nz;
    for (int q = threadIdx.x; q < cells; q += blockDim.x) {
      const int a = q / (ny * nz), rem = q - a * (ny * nz), b = rem / nz;
      int i = c0[0] + a, j = c0[1] + b, k = c0[2] + (rem - b * nz);
      if (P.per[0]) i = wrapc(i, P.cn[0]);
      if (P.per[1]) j = wrapc(j, P.cn[1]);
      if (P.per[2]) k = wrapc(k, P.cn[2]);
      cs[q] = P.cu[(long long)i * P.cxs + (long long)j * P.cys + k];
    }
  }
  __syncthreads();
  {  // u += trilinear correction on every interior cell of the region (prolong_cell's sums)
    const T w1 = (T)0.421875, w2 = (T)0.140625, w3 = (T)0.046875, w4 = (T)0.015625;
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      lo[a] = P.per[a] ? g.r0[a] : max(g.r0[a], 0);
      hi[a] = P.per[a] ? g.r1[a] : min(g.r1[a], P.n[a]);
    }
    const int ny = hi[1] - lo[1], nz = hi[2] - lo[2], cells = (hi[0] - lo[0]) * ny * nz;
    for (int q = threadIdx.x; q < cells; q += blockDim.x) {
      const int a = q / (ny * nz), rem = q - a * (ny * nz), b = rem / nz;
      const int i = lo[0] + a, j = lo[1] + b, k = lo[2] + (rem - b * nz);
      const int pi = i >> 1, pj = j >> 1, pk = k >> 1;  // parent (floor)
      // child offsets: 0 = upper child (neighbours at +1), 1 = lower child (-1)
      const int dx = 2 * pi + 1 - i, dy = 2 * pj + 1 - j, dz = 2 * pk + 1 - k;
      const int sx = dx ? -csx : csx, sy = dy ? -csy : csy, sz = dz ? -1 : 1;
      const int c = (pi - c0[0]) * csx + (pj - c0[1]) * csy + (pk - c0[2]);
      const T X = cs[c + sx], Y = cs[c + sy], Z = cs[c + sz];
      const T XY = cs[c + sx + sy], XZ = cs[c + sx + sz], YZ = cs[c + sy + sz];
      // the (-x, +y, +z) child takes its corner weight from (+1, +1, +1), as prolong_cell does
      const T XYZ = (dx == 1 && dy == 0 && dz == 0) ? cs[c + csx + csy + 1] : cs[c + sx + sy + sz];
      const int r = (i - g.r0[0]) * g.sx + (j - g.r0[1]) * g.sy + (k - g.r0[2]);
      us[r] = us[r] + w1 * cs[c] + w2 * (X + Y + Z) + w3 * (XY + XZ + YZ) + w4 * XYZ;
    }
  }
  __syncthreads();
  leg_face_ghosts<T>(P, g, us, ge);
  __syncthreads();
  leg_relax<T>(P, g, us, bs, P.passes, P.order, halo - 1, ge);
  leg_write_box<T>(P, g, us, ge);
}

template <typename T>
size_t leg_smem_bytes(bool up) {
  const size_t region = (size_t)leg_region(0) * leg_region(1) * leg_region(2);
  const size_t coarse = (size_t)leg_coarse_region(0) * leg_coarse_region(1) * leg_coarse_region(2);
  return sizeof(T) * (2 * region + (up ? coarse : 0));
}

template <typename T>
ocu_status launch_leg(const LegLevel<T> &P, bool up, cudaStream_t s) {
  if (P.passes < 2 || P.passes > 2 * kLegMaxNu || (P.passes & 1))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] launch_leg - unsupported smoothing count %d", P.passes / 2);
  const size_t bytes = leg_smem_bytes<T>(up);
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device and kernel
  int dev = 0;
  OCU_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
  const unsigned long long bit = 1ull << ((2 * dev + (up ? 1 : 0)) & 63);
  if (!(attr_set.load() & bit)) {
    OCU_TRY(check_cuda(cudaFuncSetAttribute(up ? k_leg_up<T> : k_leg_down<T>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                       "cudaFuncSetAttribute(k_leg)"));
    attr_set.fetch_or(bit);
  }
  dim3 grid((P.n[2] + leg_tile(2) - 1) / leg_tile(2), (P.n[1] + leg_tile(1) - 1) / leg_tile(1),
            (P.n[0] + leg_tile(0) - 1) / leg_tile(0));
  if (up) launch_pdl(k_leg_up<T>, grid, kLegThreads, bytes, s, P);
  else launch_pdl(k_leg_down<T>, grid, kLegThreads, bytes, s, P);
  return check_launch(up ? "k_leg_up" : "k_leg_down");
}

template ocu_status launch_leg<float>(const LegLevel<float> &, bool, cudaStream_t);
template ocu_status launch_leg<double>(const LegLevel<double> &, bool, cudaStream_t);

}  // namespace ocub
