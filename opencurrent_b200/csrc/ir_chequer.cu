// FP32 correction solver of the refinement mixed solve on the red/black split layout (see
// ir_chequer.h).  This is the library's own inner solver, not a reference routine: its operator,
// smoother and transfer operators are the reference multigrid's (7-point operator with the
// reference's boundary diagonal modifications, Yavneh-omega red-black SOR, 8-cell restriction,
// trilinear prolongation; sol_mgpressure3ddevf.cu:38-252), evaluated with fused multiply-adds
// and a precomputed omega/diagonal, and checked against an FP64 multigrid solution instead of
// bit for bit.
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "ir_chequer.h"
#include "mg_fused.h"

namespace ocub {

namespace {

// Homogeneous boundary rules of the correction equation, face order xpos, xneg, ypos, yneg,
// zpos, zneg: the value read across a Neumann face is the cell's own value, across a
// Dirichlet face its negation, across a face with no condition zero; periodic axes wrap.  The
// diagonal modifications are the reference's (sol_mgpressure3d.cpp:49-64): Neumann -f,
// Dirichlet +f.
struct ChqBC {
  float sxp, sxn, syp, syn, szp, szn;
  float mxp, mxn, myp, myn, mzp, mzn;
  int px, py, pz;
};

// One level's operator and smoother coefficients.
struct ChqK {
  float c0, c1;            // 1 - omega, omega / ld
  float omega, ld, hsq;    // boundary cells: u + omega * (t - ld u) / (ld + mod)
  float fx, fy, fz;
  float fxh, fyh, fzh, dgh;  // residual: f / h^2, ld / h^2
};

struct ChqG {
  float *u0, *u1, *b0, *b1;
  int nx, ny, nz, rz;
  int qsh, ysh, zsh;  // log2 of rz/4, ny, nz when powers of two, else -1
};

int log2_exact(int v) {
  if (v <= 0 || (v & (v - 1))) return -1;
  int s = 0;
  while ((1 << s) < v) s++;
  return s;
}

float sgn_of(const ocu_bc &b) {
  if (b.type == OCU_BC_NEUMANN) return 1.f;
  if (b.type == OCU_BC_DIRICHELET) return -1.f;
  return 0.f;
}

__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ float4 scale4(float4 a, float s) { return make_float4(s * a.x, s * a.y, s * a.z, s * a.w); }

// New value of one cell: t = sum_a f_a (left_a + right_a) - h^2 b; interior cells
// (1 - omega) u + omega/ld t, boundary cells u + omega (t - ld u) / (ld + mod).
__device__ __forceinline__ float relax_cell(float u, float b, float sx, float sy, float sz, const ChqK &k,
                                            float mod) {
  const float t = __fmaf_rn(k.fz, sz, __fmaf_rn(k.fy, sy, __fmaf_rn(k.fx, sx, -k.hsq * b)));
  if (mod == 0.f) return __fmaf_rn(k.c1, t, k.c0 * u);
  return __fmaf_rn(k.omega / (k.ld + mod), __fmaf_rn(-k.ld, u, t), u);
}

__device__ __forceinline__ float residual_cell(float u, float b, float sx, float sy, float sz, const ChqK &k) {
  return b - __fmaf_rn(k.fzh, sz, __fmaf_rn(k.fyh, sy, __fmaf_rn(k.fxh, sx, -k.dgh * u)));
}

__device__ __forceinline__ void split_index(int t, int div, int sh, int &quot, int &rem) {
  if (sh >= 0) {
    quot = t >> sh;
    rem = t & (div - 1);
  } else {
    quot = t / div;
    rem = t - quot * div;
  }
}

// One colour of a red-black SOR iteration.  A thread owns four consecutive entries m of one
// colour row (one float4); the z neighbours are the other colour's entries m - 1 + p .. m + p
// of the same row (p = row parity of this colour), the x and y neighbours its entries m of the
// four neighbouring rows.
// Launch shapes, measured at 256^3 with CUDA events on back-to-back launches: the colour sweep
// in blocks of 128 (one iteration 49.9 us against 51.4 with 256 and 62.1 with 512 threads), the
// restriction and the prolongation capped at 64 registers for four blocks of 256 per SM
// (restriction 45.1 us against 49.0 at three blocks and 61.6 at two; prolongation 36.7 us
// against 42.6 uncapped).
#ifndef CHQ_RELAX_THREADS
#define CHQ_RELAX_THREADS 128
#endif
#ifndef CHQ_RESTRICT_MINB
#define CHQ_RESTRICT_MINB 4
#endif
#ifndef CHQ_PROLONG_MINB
#define CHQ_PROLONG_MINB 4
#endif
__global__ void __launch_bounds__(CHQ_RELAX_THREADS) k_chq_relax(ChqG g, ChqK k, ChqBC bc, int color) {
  pdl_entry();
  const int qpr = g.rz >> 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)g.nx * g.ny * qpr) return;
  int row, q, i, j;
  split_index((int)t, qpr, g.qsh, row, q);
  split_index(row, g.ny, g.ysh, i, j);
  const int p = (i + j + color) & 1;
  const float *__restrict__ o = color ? g.u0 : g.u1;
  float *__restrict__ u = color ? g.u1 : g.u0;
  const float *__restrict__ bb = color ? g.b1 : g.b0;
  const long long rs = (long long)row * g.rz;
  const long long base = rs + 4 * q;
  const long long xs = (long long)g.ny * g.rz;
  const float4 U = *reinterpret_cast<const float4 *>(u + base);
  const float4 B = *reinterpret_cast<const float4 *>(bb + base);
  const float4 O = ldg4(o + base);
  float4 XM, XP, YM, YP;
  if (i > 0) XM = ldg4(o + base - xs);
  else XM = bc.px ? ldg4(o + base + (long long)(g.nx - 1) * xs) : scale4(U, bc.sxn);
  if (i < g.nx - 1) XP = ldg4(o + base + xs);
  else XP = bc.px ? ldg4(o + base - (long long)(g.nx - 1) * xs) : scale4(U, bc.sxp);
  if (j > 0) YM = ldg4(o + base - g.rz);
  else YM = bc.py ? ldg4(o + base + (long long)(g.ny - 1) * g.rz) : scale4(U, bc.syn);
  if (j < g.ny - 1) YP = ldg4(o + base + g.rz);
  else YP = bc.py ? ldg4(o + base - (long long)(g.ny - 1) * g.rz) : scale4(U, bc.syp);
  float oprev = 0.f, onext = 0.f;
  if (p == 0) {
    if (q > 0) oprev = __ldg(o + base - 1);
  } else if (8 * q + 8 < g.nz) {
    onext = __ldg(o + base + 4);
  }
  float mrow = 0.f;
  if (i == 0) mrow += bc.mxn;
  if (i == g.nx - 1) mrow += bc.mxp;
  if (j == 0) mrow += bc.myn;
  if (j == g.ny - 1) mrow += bc.myp;
  const float uo[4] = {U.x, U.y, U.z, U.w}, bo[4] = {B.x, B.y, B.z, B.w};
  const float ov[4] = {O.x, O.y, O.z, O.w};
  const float sx[4] = {XM.x + XP.x, XM.y + XP.y, XM.z + XP.z, XM.w + XP.w};
  const float sy[4] = {YM.x + YP.x, YM.y + YP.y, YM.z + YP.z, YM.w + YP.w};
  float res[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int kk = 8 * q + 2 * e + p;
    res[e] = uo[e];
    if (kk < g.nz) {
      float zm = p == 0 ? (e == 0 ? oprev : ov[(e + 3) & 3]) : ov[e];
      float zp = p == 0 ? ov[e] : (e == 3 ? onext : ov[(e + 1) & 3]);
      float mod = mrow;
      if (kk == 0) {
        zm = bc.pz ? __ldg(o + rs + (g.nz / 2 - 1)) : bc.szn * uo[e];
        mod += bc.mzn;
      }
      if (kk == g.nz - 1) {
        zp = bc.pz ? __ldg(o + rs) : bc.szp * uo[e];
        mod += bc.mzp;
      }
      res[e] = relax_cell(uo[e], bo[e], sx[e], sy[e], zm + zp, k, mod);
    }
  }
  *reinterpret_cast<float4 *>(u + base) = make_float4(res[0], res[1], res[2], res[3]);
}

// A fine row (x, y) of parity s = (x+y)&1 seen by a coarse pair: the fine cells k = 4m' + e,
// e = 0..3, are entries 2m' (e = 0, 2 -> .x, .y of colour s) and 2m' + 1 of the two colour
// arrays: e = 0: s.x, e = 1: (s^1).x, e = 2: s.y, e = 3: (s^1).y.
struct FRow {
  const float *a, *o;  // colour s and colour s^1 arrays at the row start
};

__device__ __forceinline__ FRow fine_row(const float *c0, const float *c1, const ChqG &g, int x, int y) {
  const long long id = ((long long)x * g.ny + y) * g.rz;
  const bool s = (x + y) & 1;
  FRow r;
  r.a = (s ? c1 : c0) + id;
  r.o = (s ? c0 : c1) + id;
  return r;
}

// the four cells k = 4m'..4m'+3 of a fine row
__device__ __forceinline__ void load4(const FRow &r, int m2, float v[4]) {
  const float2 A = __ldg(reinterpret_cast<const float2 *>(r.a + m2));
  const float2 O = __ldg(reinterpret_cast<const float2 *>(r.o + m2));
  v[0] = A.x; v[1] = O.x; v[2] = A.y; v[3] = O.y;
}

// Residual of the sixteen children of a coarse pair (coarse cells K = 2m', 2m' + 1 of coarse
// row (I, J)), restricted (the mean of each cell's eight) into the coarse right-hand side; the
// coarse pair's u is zeroed (the next V-cycle leg starts from zero).  All lanes of a warp share
// (I, J), so every row and boundary decision is uniform across the warp.
__global__ void __launch_bounds__(256, CHQ_RESTRICT_MINB) k_chq_restrict(ChqG f, ChqG c, ChqK k, ChqBC bc, int cm, int cmsh) {
  pdl_entry();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)c.nx * c.ny * cm) return;
  int r, mp, I, J;
  split_index((int)t, cm, cmsh, r, mp);
  split_index(r, c.ny, c.ysh, I, J);
  const int x0 = 2 * I, y0 = 2 * J, m2 = 2 * mp;
  const bool second = 2 * mp + 1 < c.nz;  // coarse K = 2m' + 1 exists
  float u[2][2][6], bv[2][2][4];           // u[a][b][1 + e], e = -1..4
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++) {
      const FRow R = fine_row(f.u0, f.u1, f, x0 + a, y0 + b);
      const FRow RB = fine_row(f.b0, f.b1, f, x0 + a, y0 + b);
      float v[4];
      load4(R, m2, v);
#pragma unroll
      for (int e = 0; e < 4; e++) u[a][b][1 + e] = v[e];
      load4(RB, m2, bv[a][b]);
      // k = 4m' - 1: colour s^1 entry 2m' - 1; k = 4m' + 4: colour s entry 2m' + 2
      if (mp > 0) u[a][b][0] = __ldg(R.o + m2 - 1);
      else u[a][b][0] = bc.pz ? __ldg(R.o + f.nz / 2 - 1) : bc.szn * u[a][b][1];
      if (4 * mp + 4 < f.nz) u[a][b][5] = __ldg(R.a + m2 + 2);
      else u[a][b][5] = bc.pz ? __ldg(R.a) : bc.szp * u[a][b][4];
      // an odd coarse row ends on K = 2m': the fine row ends on k = 4m' + 1 (its z+ neighbour is
      // the boundary value); k = 4m' + 2, 4m' + 3 are padding and their residuals unused
      if (!second) u[a][b][3] = bc.szp * u[a][b][2];
    }
  // rows around the 2x2 block of child rows: xo[side][b][e], yo[a][side][e]
  float xo[2][2][4], yo[2][2][4];
#pragma unroll
  for (int b = 0; b < 2; b++) {
    const int y = y0 + b;
    if (x0 > 0 || bc.px) load4(fine_row(f.u0, f.u1, f, x0 > 0 ? x0 - 1 : f.nx - 1, y), m2, xo[0][b]);
    else
#pragma unroll
      for (int e = 0; e < 4; e++) xo[0][b][e] = bc.sxn * u[0][b][1 + e];
    if (x0 + 2 < f.nx || bc.px) load4(fine_row(f.u0, f.u1, f, x0 + 2 < f.nx ? x0 + 2 : 0, y), m2, xo[1][b]);
    else
#pragma unroll
      for (int e = 0; e < 4; e++) xo[1][b][e] = bc.sxp * u[1][b][1 + e];
  }
#pragma unroll
  for (int a = 0; a < 2; a++) {
    const int x = x0 + a;
    if (y0 > 0 || bc.py) load4(fine_row(f.u0, f.u1, f, x, y0 > 0 ? y0 - 1 : f.ny - 1), m2, yo[a][0]);
    else
#pragma unroll
      for (int e = 0; e < 4; e++) yo[a][0][e] = bc.syn * u[a][0][1 + e];
    if (y0 + 2 < f.ny || bc.py) load4(fine_row(f.u0, f.u1, f, x, y0 + 2 < f.ny ? y0 + 2 : 0), m2, yo[a][1]);
    else
#pragma unroll
      for (int e = 0; e < 4; e++) yo[a][1][e] = bc.syp * u[a][1][1 + e];
  }
  float sum[2] = {0.f, 0.f};
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const float xm = a ? u[0][b][1 + e] : xo[0][b][e];
        const float xp = a ? xo[1][b][e] : u[1][b][1 + e];
        const float ym = b ? u[a][0][1 + e] : yo[a][0][e];
        const float yp = b ? yo[a][1][e] : u[a][1][1 + e];
        sum[e >> 1] += residual_cell(u[a][b][1 + e], bv[a][b][e], xm + xp, ym + yp, u[a][b][e] + u[a][b][2 + e], k);
      }
  // coarse row parity sc: K = 2m' is colour sc entry m', K = 2m' + 1 colour sc^1 entry m'
  const long long cid = ((long long)I * c.ny + J) * c.rz + mp;
  const bool sc = (I + J) & 1;
  (sc ? c.b1 : c.b0)[cid] = 0.125f * sum[0];
  (sc ? c.u1 : c.u0)[cid] = 0.f;
  if (second) {
    (sc ? c.b0 : c.b1)[cid] = 0.125f * sum[1];
    (sc ? c.u0 : c.u1)[cid] = 0.f;
  }
}

// Trilinear prolongation (weights 27, 9, 3, 1 / 64) of a coarse pair (K = 2m', 2m' + 1 of coarse
// row (I, J)) into its sixteen children, added to the fine u.  Coarse values outside the domain
// follow the homogeneous rules axis by axis (a corner is the product of the face signs times the
// cell).  Rows are warp-uniform; the eight fine float2 pairs are loaded before the first store.
__global__ void __launch_bounds__(256, CHQ_PROLONG_MINB) k_chq_prolong(ChqG c, ChqG f, ChqBC bc, int cm, int cmsh) {
  pdl_entry();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)c.nx * c.ny * cm) return;
  int r, mp, I, J;
  split_index((int)t, cm, cmsh, r, mp);
  split_index(r, c.ny, c.ysh, I, J);
  const int K0 = 2 * mp;
  const bool second = K0 + 1 < c.nz;
  // V[di][dj][q]: coarse value at (I + di - 1, J + dj - 1, K0 - 1 + q), q = 0..3
  float V[3][3][4];
#pragma unroll
  for (int di = 0; di < 3; di++)
#pragma unroll
    for (int dj = 0; dj < 3; dj++) {
      int x = I + di - 1, y = J + dj - 1;
      float sg = 1.f;
      if (x < 0) { if (bc.px) x = c.nx - 1; else { x = I; sg = bc.sxn; } }
      else if (x >= c.nx) { if (bc.px) x = 0; else { x = I; sg = bc.sxp; } }
      if (y < 0) { if (bc.py) y = c.ny - 1; else { y = J; sg *= bc.syn; } }
      else if (y >= c.ny) { if (bc.py) y = 0; else { y = J; sg *= bc.syp; } }
      const FRow R = fine_row(c.u0, c.u1, c, x, y);  // colour s' (K even) / s'^1 (K odd)
      const float v0 = __ldg(R.a + mp);
      const float v1 = second ? __ldg(R.o + mp) : (bc.pz ? __ldg(R.a) : bc.szp * v0);
      float vm, vp;
      if (mp > 0) vm = __ldg(R.o + mp - 1);
      else vm = bc.pz ? __ldg(R.o + c.nz / 2 - 1) : bc.szn * v0;
      if (K0 + 2 < c.nz) vp = __ldg(R.a + mp + 1);
      else vp = bc.pz ? __ldg(R.a) : bc.szp * v1;
      V[di][dj][0] = sg * vm;
      V[di][dj][1] = sg * v0;
      V[di][dj][2] = sg * v1;
      V[di][dj][3] = sg * vp;
    }
  float2 *dA[2][2], *dO[2][2];
  float2 fa[2][2], fo[2][2];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++) {
      const FRow R = fine_row(f.u0, f.u1, f, 2 * I + a, 2 * J + b);
      dA[a][b] = reinterpret_cast<float2 *>(const_cast<float *>(R.a) + 2 * mp);
      dO[a][b] = reinterpret_cast<float2 *>(const_cast<float *>(R.o) + 2 * mp);
      fa[a][b] = *dA[a][b];
      fo[a][b] = *dO[a][b];
    }
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++) {
      const int ea = a ? 2 : 0, eb = b ? 2 : 0;
      float out[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        // fine k = 4m' + e is a child of coarse q = 1 + (e >> 1) on its side sz (e even: -1)
        const int q = 1 + (e >> 1), qz = (e & 1) ? q + 1 : q - 1;
        const float s1 = V[ea][1][q] + V[1][eb][q] + V[1][1][qz];
        const float s2 = V[ea][eb][q] + V[ea][1][qz] + V[1][eb][qz];
        out[e] = __fmaf_rn(27.f, V[1][1][q], __fmaf_rn(9.f, s1, __fmaf_rn(3.f, s2, V[ea][eb][qz])));
      }
      float2 A = fa[a][b], O = fo[a][b];
      A.x = __fmaf_rn(out[0], 0.015625f, A.x);
      O.x = __fmaf_rn(out[1], 0.015625f, O.x);
      if (second) {
        A.y = __fmaf_rn(out[2], 0.015625f, A.y);
        O.y = __fmaf_rn(out[3], 0.015625f, O.y);
      }
      *dA[a][b] = A;
      *dO[a][b] = O;
    }
}

__global__ void k_chq_zero(float *p, long long n) {
  pdl_entry();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) p[q] = 0.f;
}

// ---- the small levels in one CTA ------------------------------------------------------------
// Levels s..L-1 of the hierarchy staged in shared memory (four colour arrays per level) and
// worked through by one thread block, the phases separated by __syncthreads: a colour sweep (one
// cell per thread and trip), a residual (one fine cell per trip, into a scratch array), its
// restriction (the eight-cell sum, one coarse cell per trip), a prolongation (one fine cell per
// trip).  Cells are decoded with shifts when the sizes are powers of two, and cells away from
// every face read their neighbours without boundary tests, so a phase over a small level is a
// short chain per thread.
constexpr int kChqMaxTail = 8;

struct SLv {
  int nx, ny, nz, rz;
  int off;                   // first float of the level's four arrays in shared memory
  int mlog, ylog, nzlog;     // log2 of M = ceil(nz/2), ny, nz when powers of two, else -1
  ChqK k;
  float *gu0, *gu1, *gb0, *gb1;  // the level's global arrays
};

struct ChqTail {
  SLv lv[kChqMaxTail];
  int nlev;         // levels s..L-1 held here (lv[0] = level s)
  int nu1, nu2, citers;
  int level0;       // whether lv[0] is level 0 of the hierarchy (no post-smoothing there)
  int fmg;          // 1: FMG from lv[0]'s right-hand side (u starts at zero); 0: one V-cycle
  int scratch;      // first float of the residual scratch (2 * nx * ny * rz of the largest
                    // level that is restricted)
  ChqBC bc;
};

struct SG {
  float *u0, *u1, *b0, *b1;
  int nx, ny, nz, rz, M, mlog, ylog, nzlog;
};

__device__ __forceinline__ SG sg_of(const SLv &l, float *sm) {
  const int n = l.nx * l.ny * l.rz;
  SG g;
  g.u0 = sm + l.off; g.u1 = g.u0 + n; g.b0 = g.u0 + 2 * n; g.b1 = g.u0 + 3 * n;
  g.nx = l.nx; g.ny = l.ny; g.nz = l.nz; g.rz = l.rz; g.M = (l.nz + 1) >> 1;
  g.mlog = l.mlog; g.ylog = l.ylog; g.nzlog = l.nzlog;
  return g;
}

__device__ __forceinline__ void dec(int q, int d, int lg, int &hi, int &lo) {
  if (lg >= 0) { hi = q >> lg; lo = q & (d - 1); }
  else { hi = q / d; lo = q - hi * d; }
}

// entry of cell (i, j, k) (inside the domain)
__device__ __forceinline__ int s_id(const SG &g, int i, int j, int k) { return (i * g.ny + j) * g.rz + (k >> 1); }
// colour arrays by a run-time colour (selects: indexing a small array member with a run-time
// value would put the struct in local memory)
__device__ __forceinline__ float *s_ucol(const SG &g, int c) { return c ? g.u1 : g.u0; }
__device__ __forceinline__ float *s_bcol(const SG &g, int c) { return c ? g.b1 : g.b0; }


// Neighbour sums of cell (i, j, k), whose entry in its colour array is id (the same entry of the
// other colour's array o holds its x and y neighbours in the neighbouring rows); uv is its value.
// Faces apply the homogeneous rules with selects (the same as the level kernels).
__device__ __forceinline__ void s_sums(const SG &g, const ChqBC &bc, int i, int j, int k, int id, const float *o,
                                       float uv, float &sx, float &sy, float &sz) {
  const int xs = g.ny * g.rz, rs = id - (k >> 1);
  const float xm = i > 0 ? o[id - xs] : (bc.px ? o[id + (g.nx - 1) * xs] : bc.sxn * uv);
  const float xp = i < g.nx - 1 ? o[id + xs] : (bc.px ? o[id - (g.nx - 1) * xs] : bc.sxp * uv);
  const float ym = j > 0 ? o[id - g.rz] : (bc.py ? o[id + (g.ny - 1) * g.rz] : bc.syn * uv);
  const float yp = j < g.ny - 1 ? o[id + g.rz] : (bc.py ? o[id - (g.ny - 1) * g.rz] : bc.syp * uv);
  const float zm = k > 0 ? o[rs + ((k - 1) >> 1)] : (bc.pz ? o[rs + ((g.nz - 1) >> 1)] : bc.szn * uv);
  const float zp = k < g.nz - 1 ? o[rs + ((k + 1) >> 1)] : (bc.pz ? o[rs] : bc.szp * uv);
  sx = xm + xp;
  sy = ym + yp;
  sz = zm + zp;
}

__device__ __forceinline__ float s_mod(const SG &g, const ChqBC &bc, int i, int j, int k) {
  float mod = 0.f;
  if (i == 0) mod += bc.mxn;
  if (i == g.nx - 1) mod += bc.mxp;
  if (j == 0) mod += bc.myn;
  if (j == g.ny - 1) mod += bc.myp;
  if (k == 0) mod += bc.mzn;
  if (k == g.nz - 1) mod += bc.mzp;
  return mod;
}

__device__ void s_relax(const SG &g, const ChqK &kk, const ChqBC &bc, int color) {
  const int cells = g.nx * g.ny * g.M;
  float *u = s_ucol(g, color);
  const float *b = s_bcol(g, color), *o = s_ucol(g, color ^ 1);
  for (int q = threadIdx.x; q < cells; q += blockDim.x) {
    int row, m, i, j;
    dec(q, g.M, g.mlog, row, m);
    dec(row, g.ny, g.ylog, i, j);
    const int k = 2 * m + ((i + j + color) & 1);
    if (k >= g.nz) continue;
    const int id = row * g.rz + m;
    const float uv = u[id];
    float sx, sy, sz;
    s_sums(g, bc, i, j, k, id, o, uv, sx, sy, sz);
    u[id] = relax_cell(uv, b[id], sx, sy, sz, kk, s_mod(g, bc, i, j, k));
  }
}

// residual of every cell of level g into r (colour arrays r[0], r[1] laid out like u)
__device__ void s_residual(const SG &g, const ChqK &kk, const ChqBC &bc, float *r0, float *r1) {
  const int cells = g.nx * g.ny * g.nz;
  for (int q = threadIdx.x; q < cells; q += blockDim.x) {
    int row, k, i, j;
    dec(q, g.nz, g.nzlog, row, k);
    dec(row, g.ny, g.ylog, i, j);
    const int col = (i + j + k) & 1, id = row * g.rz + (k >> 1);
    const float uv = s_ucol(g, col)[id];
    float sx, sy, sz;
    s_sums(g, bc, i, j, k, id, s_ucol(g, col ^ 1), uv, sx, sy, sz);
    (col ? r1 : r0)[id] = residual_cell(uv, s_bcol(g, col)[id], sx, sy, sz, kk);
  }
}

// coarse b = mean of the eight children's residuals, coarse u = 0
__device__ void s_restrict_sum(const SG &f, const SG &c, const float *r0, const float *r1) {
  const int cells = c.nx * c.ny * c.nz;
  for (int q = threadIdx.x; q < cells; q += blockDim.x) {
    int row, K, I, J;
    dec(q, c.nz, c.nzlog, row, K);
    dec(row, c.ny, c.ylog, I, J);
    float sum = 0.f;
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 2; b++) {
        // children k = 2K (colour (a+b)&1) and 2K + 1 (the other), both at entry K of the row
        const int id = ((2 * I + a) * f.ny + 2 * J + b) * f.rz + K;
        sum += r0[id] + r1[id];
      }
    const int col = (I + J + K) & 1, cid = row * c.rz + (K >> 1);
    s_bcol(c, col)[cid] = 0.125f * sum;
    s_ucol(c, col)[cid] = 0.f;
  }
}

// the coarse neighbour index along one axis of a fine cell's parent, with the face rule's sign
__device__ __forceinline__ int s_nbr(int I, int d, int n, bool per, float sneg, float spos, float &sg) {
  const int I2 = I + d;
  if (I2 < 0) { if (per) return n - 1; sg = sneg; return I; }
  if (I2 >= n) { if (per) return 0; sg = spos; return I; }
  return I2;
}

// trilinear prolongation into every fine cell
__device__ void s_prolong(const SG &c, const SG &f, const ChqBC &bc) {
  const int cells = f.nx * f.ny * f.nz;
  for (int q = threadIdx.x; q < cells; q += blockDim.x) {
    int row, k, i, j;
    dec(q, f.nz, f.nzlog, row, k);
    dec(row, f.ny, f.ylog, i, j);
    const int I = i >> 1, J = j >> 1, K = k >> 1;
    float gx = 1.f, gy = 1.f, gz = 1.f;
    const int I2 = s_nbr(I, (i & 1) ? 1 : -1, c.nx, bc.px, bc.sxn, bc.sxp, gx);
    const int J2 = s_nbr(J, (j & 1) ? 1 : -1, c.ny, bc.py, bc.syn, bc.syp, gy);
    const int K2 = s_nbr(K, (k & 1) ? 1 : -1, c.nz, bc.pz, bc.szn, bc.szp, gz);
    auto cv = [&](int x, int y, int z) { return s_ucol(c, (x + y + z) & 1)[(x * c.ny + y) * c.rz + (z >> 1)]; };
    const float c000 = cv(I, J, K);
    const float s1 = gx * cv(I2, J, K) + gy * cv(I, J2, K) + gz * cv(I, J, K2);
    const float s2 = gx * gy * cv(I2, J2, K) + gx * gz * cv(I2, J, K2) + gy * gz * cv(I, J2, K2);
    const float s3 = gx * gy * gz * cv(I2, J2, K2);
    const float v = __fmaf_rn(27.f, c000, __fmaf_rn(9.f, s1, __fmaf_rn(3.f, s2, s3)));
    float *u = s_ucol(f, (i + j + k) & 1);
    const int id = row * f.rz + (k >> 1);
    u[id] = __fmaf_rn(v, 0.015625f, u[id]);
  }
}

__device__ void s_relax_iters(const SG &g, const ChqK &kk, const ChqBC &bc, int iterations) {
  for (int it = 0; it < iterations; it++)
    for (int color = 0; color < 2; color++) {
      s_relax(g, kk, bc, color);
      __syncthreads();
    }
}

// The phases read the level table from shared memory (a copy of the launch parameters made
// with constant indices: indexing the parameter array with a run-time level would give every
// thread a local-memory copy of it).
__device__ void s_restrict(const ChqTail &T, const SLv *lv, float *sm, int l) {
  const SG f = sg_of(lv[l], sm), c = sg_of(lv[l + 1], sm);
  float *r0 = sm + T.scratch, *r1 = r0 + f.nx * f.ny * f.rz;
  s_residual(f, lv[l].k, T.bc, r0, r1);
  __syncthreads();
  s_restrict_sum(f, c, r0, r1);
  __syncthreads();
}

// one V-cycle from tail level a (0-based within the tail)
__device__ void s_vcycle(const ChqTail &T, const SLv *lv, float *sm, int a) {
  const int last = T.nlev - 1;
  for (int l = a; l < last; l++) {
    s_relax_iters(sg_of(lv[l], sm), lv[l].k, T.bc, T.nu1);
    s_restrict(T, lv, sm, l);
  }
  s_relax_iters(sg_of(lv[last], sm), lv[last].k, T.bc, T.citers);
  for (int l = last - 1; l >= a; l--) {
    s_prolong(sg_of(lv[l + 1], sm), sg_of(lv[l], sm), T.bc);
    __syncthreads();
    if (!(l == 0 && T.level0)) s_relax_iters(sg_of(lv[l], sm), lv[l].k, T.bc, T.nu2);
  }
}

__global__ void __launch_bounds__(1024) k_chq_tail(ChqTail T) {
  pdl_entry();
  extern __shared__ float sm[];
  __shared__ SLv lv[kChqMaxTail];
  if (threadIdx.x == 0) {
#pragma unroll
    for (int l = 0; l < kChqMaxTail; l++)
      if (l < T.nlev) lv[l] = T.lv[l];
  }
  __syncthreads();
  const SLv &L0 = lv[0];
  const int n0 = L0.nx * L0.ny * L0.rz;
  float *g0 = sm + L0.off;
  for (int q = threadIdx.x; q < n0; q += blockDim.x) {
    g0[q] = T.fmg ? 0.f : L0.gu0[q];
    g0[n0 + q] = T.fmg ? 0.f : L0.gu1[q];
    g0[2 * n0 + q] = L0.gb0[q];
    g0[3 * n0 + q] = L0.gb1[q];
  }
  // the coarser levels (their padding entries stay zero)
  for (int l = 1; l < T.nlev; l++) {
    const int n = 4 * lv[l].nx * lv[l].ny * lv[l].rz;
    for (int q = threadIdx.x; q < n; q += blockDim.x) sm[lv[l].off + q] = 0.f;
  }
  __syncthreads();
  if (T.fmg) {
    for (int l = 0; l < T.nlev - 1; l++) s_restrict(T, lv, sm, l);
    const int last = T.nlev - 1;
    s_relax_iters(sg_of(lv[last], sm), lv[last].k, T.bc, T.citers);
    for (int f = last - 1; f >= 0; f--) {
      s_prolong(sg_of(lv[f + 1], sm), sg_of(lv[f], sm), T.bc);
      __syncthreads();
      s_vcycle(T, lv, sm, f);
    }
  } else {
    s_vcycle(T, lv, sm, 0);
  }
  for (int q = threadIdx.x; q < n0; q += blockDim.x) {
    L0.gu0[q] = g0[q];
    L0.gu1[q] = g0[n0 + q];
  }
}

// FP64 residual of the refinement step, written as float into the level-0 colour arrays, with
// per-row sum of squares and max |r| (one warp per row (i, j)).
struct OuterCoef {
  double fxh, fyh, fzh, dg;
};

template <bool VEC>
__global__ void __launch_bounds__(256) k_chq_outer_residual(const double *__restrict__ x, const double *__restrict__ b,
                                                            long long xs, long long ys, int nx, int ny, int nz,
                                                            OuterCoef c, float *__restrict__ B0,
                                                            float *__restrict__ B1, int rz,
                                                            double *__restrict__ rows2,
                                                            double *__restrict__ rowsinf) {
  pdl_entry();
  const int lane = threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (j >= ny) return;  // whole warp
  const long long row = (long long)i * xs + (long long)j * ys;
  const long long crow = ((long long)i * ny + j) * rz;
  const bool s = (i + j) & 1;
  float *__restrict__ Bs = s ? B1 : B0;
  float *__restrict__ Bo = s ? B0 : B1;
  double acc2 = 0, accinf = 0;
  for (int m = lane; 2 * m < nz; m += 32) {
    if (VEC) {  // nz even, rows on 16-byte boundaries: the pair and its neighbours as double2
      const long long id = row + 2 * m;
      const double2 X = *reinterpret_cast<const double2 *>(x + id), B = *reinterpret_cast<const double2 *>(b + id);
      const double2 YM = *reinterpret_cast<const double2 *>(x + id - ys), YP = *reinterpret_cast<const double2 *>(x + id + ys);
      const double2 XM = *reinterpret_cast<const double2 *>(x + id - xs), XP = *reinterpret_cast<const double2 *>(x + id + xs);
      const double zl = x[id - 1], zr = x[id + 2];
      const double r0 = B.x - (c.fzh * (zl + X.y) + c.fyh * (YM.x + YP.x) + c.fxh * (XM.x + XP.x) - c.dg * X.x);
      const double r1 = B.y - (c.fzh * (X.x + zr) + c.fyh * (YM.y + YP.y) + c.fxh * (XM.y + XP.y) - c.dg * X.y);
      Bs[crow + m] = (float)r0;
      Bo[crow + m] = (float)r1;
      acc2 += r0 * r0 + r1 * r1;
      accinf = fmax(accinf, fmax(fabs(r0), fabs(r1)));
      continue;
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int k = 2 * m + h;
      if (k < nz) {
        const long long id = row + k;
        const double r = b[id] - (c.fzh * (x[id - 1] + x[id + 1]) + c.fyh * (x[id - ys] + x[id + ys]) +
                                  c.fxh * (x[id - xs] + x[id + xs]) - c.dg * x[id]);
        (h ? Bo : Bs)[crow + m] = (float)r;
        acc2 += r * r;
        accinf = fmax(accinf, fabs(r));
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc2 += __shfl_down_sync(0xffffffffu, acc2, o);
    accinf = fmax(accinf, __shfl_down_sync(0xffffffffu, accinf, o));
  }
  if (lane == 0) {
    rows2[(long long)i * ny + j] = acc2;
    rowsinf[(long long)i * ny + j] = accinf;
  }
}

// x += (double) e on the interior, e on the level-0 colour arrays.
template <bool VEC>
__global__ void __launch_bounds__(256) k_chq_add_correction(double *__restrict__ x, long long xs, long long ys,
                                                            int nx, int ny, int nz, const float *__restrict__ E0,
                                                            const float *__restrict__ E1, int rz) {
  pdl_entry();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (j >= ny || 2 * m >= nz) return;
  const long long id = (long long)i * xs + (long long)j * ys + 2 * m;
  const long long cid = ((long long)i * ny + j) * rz + m;
  const bool s = (i + j) & 1;
  const float e0 = (s ? E1 : E0)[cid], e1 = (s ? E0 : E1)[cid];
  if (VEC) {
    double2 X = *reinterpret_cast<double2 *>(x + id);
    X.x = X.x + (double)e0;
    X.y = X.y + (double)e1;
    *reinterpret_cast<double2 *>(x + id) = X;
    return;
  }
  x[id] = x[id] + (double)e0;
  if (2 * m + 1 < nz) x[id + 1] = x[id + 1] + (double)e1;
}

}  // namespace

static ChqBC make_bc(const ocu_bc_set &bc, double fx, double fy, double fz) {
  ChqBC d;
  d.sxp = sgn_of(bc.xpos); d.sxn = sgn_of(bc.xneg);
  d.syp = sgn_of(bc.ypos); d.syn = sgn_of(bc.yneg);
  d.szp = sgn_of(bc.zpos); d.szn = sgn_of(bc.zneg);
  d.mxp = (float)bc_diag_mod(bc.xpos, fx); d.mxn = (float)bc_diag_mod(bc.xneg, fx);
  d.myp = (float)bc_diag_mod(bc.ypos, fy); d.myn = (float)bc_diag_mod(bc.yneg, fy);
  d.mzp = (float)bc_diag_mod(bc.zpos, fz); d.mzn = (float)bc_diag_mod(bc.zneg, fz);
  d.px = bc.xpos.type == OCU_BC_PERIODIC;
  d.py = bc.ypos.type == OCU_BC_PERIODIC;
  d.pz = bc.zpos.type == OCU_BC_PERIODIC;
  return d;
}

static ChqK make_k(double h, double fx, double fy, double fz, double omega) {
  ChqK k;
  const double ld = 2 * (fx + fy + fz);
  k.c0 = (float)(1 - omega);
  k.c1 = (float)(omega / ld);
  k.omega = (float)omega;
  k.ld = (float)ld;
  k.hsq = (float)(h * h);
  k.fx = (float)fx; k.fy = (float)fy; k.fz = (float)fz;
  k.fxh = (float)(fx / (h * h)); k.fyh = (float)(fy / (h * h)); k.fzh = (float)(fz / (h * h));
  k.dgh = (float)(ld / (h * h));
  return k;
}

static ChqG make_g(const ChqLevel &l) {
  ChqG g;
  g.u0 = l.u[0]; g.u1 = l.u[1]; g.b0 = l.b[0]; g.b1 = l.b[1];
  g.nx = l.nx; g.ny = l.ny; g.nz = l.nz; g.rz = l.rz;
  g.qsh = log2_exact(l.rz / 4);
  g.ysh = log2_exact(l.ny);
  g.zsh = log2_exact(l.nz);
  return g;
}

static int round4(int v) { return (v + 3) & ~3; }

// Shared memory of a level in the single-CTA tail: its four colour arrays.
static size_t level_smem(const std::array<int, 3> &d) {
  return (size_t)4 * d[0] * d[1] * round4((d[2] + 1) / 2) * sizeof(float);
}

// the tail's residual scratch: two colour arrays of its largest restricted level
static size_t scratch_smem(const std::array<int, 3> &d) { return level_smem(d) / 2; }

// Largest shared-memory footprint of the tail kernel (opt-in above 48 KB).
constexpr size_t kTailSmemCap = 200 * 1024;
// Levels with at most this many cells join the single-CTA tail (OCU_B200_CHQ_TAIL overrides;
// the coarsest level always runs there).  Measured at 256^3 (refinement solve, one box): 3.82 ms
// with only the coarsest level (4^3) in the tail, 3.75 ms with 8^3 too, 3.78 ms with 16^3 too --
// a tail phase over a 16^3 level costs about what a launch with programmatic dependencies does.
constexpr long long kChqTailCells = 512;

static long long tail_cells_setting() {
  const char *e = std::getenv("OCU_B200_CHQ_TAIL");
  return e ? std::atoll(e) : kChqTailCells;
}

// First level of the single-CTA tail: the largest run of coarse levels, each with at most
// tail_cells cells, whose arrays fit the shared-memory cap (at least the coarsest level).
static int tail_first(const std::vector<std::array<int, 3>> &dims, long long tail_cells) {
  const int L = (int)dims.size();
  int first = L - 1;
  size_t bytes = level_smem(dims[L - 1]);
  while (first > 0 && first - 1 >= L - kChqMaxTail) {
    const auto &d = dims[first - 1];
    const size_t b = level_smem(d);
    if ((long long)d[0] * d[1] * d[2] > tail_cells || bytes + b + scratch_smem(d) > kTailSmemCap) break;
    bytes += b;
    first--;
  }
  return first;
}

bool ChequerMG::suits(const std::vector<std::array<int, 3>> &dims, const ocu_bc_set &bc) {
  if (dims.size() < 2) return false;
  const ocu_bc *f[6] = {&bc.xpos, &bc.xneg, &bc.ypos, &bc.yneg, &bc.zpos, &bc.zneg};
  for (int q = 0; q < 6; q++) {
    const int t = f[q]->type;
    if (t != OCU_BC_NEUMANN && t != OCU_BC_DIRICHELET && t != OCU_BC_PERIODIC && t != OCU_BC_NONE) return false;
  }
  // a periodic axis must be periodic on both faces and even on every level (the colouring
  // then continues across the wrap)
  const bool per[3] = {bc.xpos.type == OCU_BC_PERIODIC, bc.ypos.type == OCU_BC_PERIODIC,
                       bc.zpos.type == OCU_BC_PERIODIC};
  const bool per_neg[3] = {bc.xneg.type == OCU_BC_PERIODIC, bc.yneg.type == OCU_BC_PERIODIC,
                           bc.zneg.type == OCU_BC_PERIODIC};
  for (int a = 0; a < 3; a++) {
    if (per[a] != per_neg[a]) return false;
    if (per[a])
      for (const auto &d : dims)
        if (d[a] % 2) return false;
  }
  for (const auto &d : dims)
    if ((long long)d[0] * d[1] * round4((d[2] + 1) / 2) / 4 >= (1LL << 31) / 8) return false;
  return level_smem(dims.back()) <= kTailSmemCap;
}

ChequerMG::~ChequerMG() {
  if (block) cudaFree(block);
}

ocu_status ChequerMG::init(const std::vector<std::array<int, 3>> &dims, const std::vector<double> &h, double fx_,
                           double fy_, double fz_, double omega_, const ocu_bc_set &bc_h) {
  fx = fx_; fy = fy_; fz = fz_; omega = omega_; bc = bc_h;
  lv.clear();
  size_t total = 0;
  for (size_t l = 0; l < dims.size(); l++) {
    ChqLevel L{};
    L.nx = dims[l][0]; L.ny = dims[l][1]; L.nz = dims[l][2];
    L.rz = round4((L.nz + 1) / 2);
    L.h = h[l];
    lv.push_back(L);
    total += 4 * (size_t)L.nx * L.ny * L.rz;
  }
  tail_s = tail_first(dims, tail_cells_setting());
  size_t tail_bytes = 0;
  for (size_t l = tail_s; l < dims.size(); l++) tail_bytes += level_smem(dims[l]);
  OCU_TRY(check_cuda(cudaFuncSetAttribute(k_chq_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTailSmemCap),
                     "cudaFuncSetAttribute (tail kernel)"));
  (void)tail_bytes;
  OCU_TRY(check_cuda(cudaMalloc(&block, total * sizeof(float)), "cudaMalloc (FP32 refinement levels)"));
  OCU_TRY(check_cuda(cudaMemset(block, 0, total * sizeof(float)), "cudaMemset"));
  float *p = (float *)block;
  for (auto &L : lv) {
    const size_t n = (size_t)L.nx * L.ny * L.rz;
    L.u[0] = p; L.u[1] = p + n; L.b[0] = p + 2 * n; L.b[1] = p + 3 * n;
    p += 4 * n;
  }
  return OCU_OK;
}

ocu_status ChequerMG::clear_u(int l, cudaStream_t s) {
  const ChqLevel &L = lv[l];
  const long long n = 2LL * L.nx * L.ny * L.rz;  // u[0] and u[1] are adjacent
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
  launch_pdl(k_chq_zero, dim3(blocks), dim3(256), 0, s, L.u[0], n);
  return check_launch("k_chq_zero");
}

ocu_status ChequerMG::relax(int l, int iterations, bool reverse, cudaStream_t s) {
  const ChqLevel &L = lv[l];
  const ChqG g = make_g(L);
  const ChqK k = make_k(L.h, fx, fy, fz, omega);
  const ChqBC b = make_bc(bc, fx, fy, fz);
  const long long threads = (long long)L.nx * L.ny * (L.rz / 4);
  const int blocks = (int)((threads + CHQ_RELAX_THREADS - 1) / CHQ_RELAX_THREADS);
  for (int it = 0; it < iterations; it++)
    for (int h = 0; h < 2; h++) {
      launch_pdl(k_chq_relax, dim3(blocks), dim3(CHQ_RELAX_THREADS), 0, s, g, k, b, reverse ? 1 - h : h);
      OCU_TRY(check_launch("k_chq_relax"));
    }
  return OCU_OK;
}

ocu_status ChequerMG::sweep_level(int l, int color, cudaStream_t s) {
  const ChqLevel &L = lv[l];
  const long long threads = (long long)L.nx * L.ny * (L.rz / 4);
  launch_pdl(k_chq_relax, dim3((unsigned)((threads + 255) / 256)), dim3(256), 0, s, make_g(L),
             make_k(L.h, fx, fy, fz, omega), make_bc(bc, fx, fy, fz), color & 1);
  return check_launch("k_chq_relax");
}

ocu_status ChequerMG::restrict_to(int l, cudaStream_t s) {
  const ChqLevel &F = lv[l], &Cl = lv[l + 1];
  const int cm = (Cl.nz + 1) / 2;  // coarse pairs per row
  const long long n = (long long)Cl.nx * Cl.ny * cm;
  launch_pdl(k_chq_restrict, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, s, make_g(F), make_g(Cl),
             make_k(F.h, fx, fy, fz, omega), make_bc(bc, fx, fy, fz), cm, log2_exact(cm));
  return check_launch("k_chq_restrict");
}

ocu_status ChequerMG::prolong_from(int l, cudaStream_t s) {
  const ChqLevel &Cl = lv[l], &F = lv[l - 1];
  const int cm = (Cl.nz + 1) / 2;
  const long long n = (long long)Cl.nx * Cl.ny * cm;
  launch_pdl(k_chq_prolong, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, s, make_g(Cl), make_g(F),
             make_bc(bc, fx, fy, fz), cm, log2_exact(cm));
  return check_launch("k_chq_prolong");
}

ocu_status ChequerMG::tail(bool fmg, int nu1, int nu2, int citers, cudaStream_t s) {
  ChqTail T{};
  const int L = levels();
  T.nlev = L - tail_s;
  T.nu1 = nu1; T.nu2 = nu2; T.citers = citers;
  T.level0 = tail_s == 0;
  T.fmg = fmg ? 1 : 0;
  T.bc = make_bc(bc, fx, fy, fz);
  int off = 0, largest = 0;
  for (int l = tail_s; l < L; l++) {
    const ChqLevel &C = lv[l];
    SLv &d = T.lv[l - tail_s];
    d.nx = C.nx; d.ny = C.ny; d.nz = C.nz; d.rz = C.rz;
    d.off = off;
    d.mlog = log2_exact((C.nz + 1) / 2);
    d.ylog = log2_exact(C.ny);
    d.nzlog = log2_exact(C.nz);
    d.k = make_k(C.h, fx, fy, fz, omega);
    d.gu0 = C.u[0]; d.gu1 = C.u[1]; d.gb0 = C.b[0]; d.gb1 = C.b[1];
    off += 4 * C.nx * C.ny * C.rz;
    if (l < L - 1 && 2 * C.nx * C.ny * C.rz > largest) largest = 2 * C.nx * C.ny * C.rz;
  }
  T.scratch = off;
  off += largest;
  // threads: enough for the largest phase of the top level, in whole warps, at most 1024
  const ChqLevel &top = lv[tail_s];
  const long long work = (long long)top.nx * top.ny * top.nz;
  const int threads = (int)std::min<long long>(1024, std::max<long long>(64, ((work + 31) / 32) * 32));
  launch_pdl(k_chq_tail, dim3(1), dim3(threads), (size_t)off * sizeof(float), s, T);
  return check_launch("k_chq_tail");
}

// Nested iteration + V-cycles: the right-hand side restricted down to the tail, the tail
// levels solved in one launch, then on the way up each level gets the prolonged coarse solution
// and ramp_iters red-black iterations (no V-cycle: measured at 256^3, a refinement solve takes
// 3.87 ms this way against 4.61 ms with one V-cycle per ramp level, at the same residual after
// the same two refinement steps), and level 0 gets `cycles` V-cycles.
ocu_status ChequerMG::enqueue_fmg(int nu1, int nu2, int cycles, int coarse_iters, int ramp_iters, cudaStream_t s) {
  const int ts = tail_s;
  if (ts > 0) OCU_TRY(clear_u(0, s));
  for (int l = 0; l < ts; l++) OCU_TRY(restrict_to(l, s));
  OCU_TRY(tail(true, nu1, nu2, coarse_iters, s));
  if (ts == 0) {
    for (int c = 1; c < cycles; c++) OCU_TRY(tail(false, nu1, nu2, coarse_iters, s));
    return OCU_OK;
  }
  for (int f = ts - 1; f >= 1; f--) {
    OCU_TRY(prolong_from(f + 1, s));
    OCU_TRY(relax(f, ramp_iters, false, s));
  }
  OCU_TRY(prolong_from(1, s));
  for (int c = 0; c < cycles; c++) {
    for (int l = 0; l < ts; l++) {
      OCU_TRY(relax(l, nu1, false, s));
      OCU_TRY(restrict_to(l, s));
    }
    OCU_TRY(tail(false, nu1, nu2, coarse_iters, s));
    for (int l = ts - 1; l >= 0; l--) {
      OCU_TRY(prolong_from(l + 1, s));
      if (l > 0) OCU_TRY(relax(l, nu2, false, s));
    }
  }
  return OCU_OK;
}

// the FP64 grid's pairs (k, k+1), k even, are 16-byte aligned double2
static bool vec_ok(const ocu_layout &L) {
  return L.nz % 2 == 0 && L.shift % 2 == 0 && L.xstride % 2 == 0 && L.ystride % 2 == 0;
}

ocu_status ChequerMG::enqueue_residual(const double *x, const double *b, const ocu_layout &L, double h, double fx_,
                                       double fy_, double fz_, double *rows2, double *rowsinf, cudaStream_t s) {
  const ChqLevel &C0 = lv[0];
  OuterCoef c;
  c.fxh = fx_ / (h * h);
  c.fyh = fy_ / (h * h);
  c.fzh = fz_ / (h * h);
  c.dg = 2 * (fx_ + fy_ + fz_) / (h * h);
  dim3 block(32, 8), grid(1, (L.ny + 7) / 8, L.nx);
  if (vec_ok(L))
    launch_pdl(k_chq_outer_residual<true>, grid, block, 0, s, x, b, (long long)L.xstride, (long long)L.ystride, L.nx,
               L.ny, L.nz, c, C0.b[0], C0.b[1], C0.rz, rows2, rowsinf);
  else
    launch_pdl(k_chq_outer_residual<false>, grid, block, 0, s, x, b, (long long)L.xstride, (long long)L.ystride, L.nx,
               L.ny, L.nz, c, C0.b[0], C0.b[1], C0.rz, rows2, rowsinf);
  return check_launch("k_chq_outer_residual");
}

ocu_status ChequerMG::enqueue_add_correction(double *x, const ocu_layout &L, cudaStream_t s) {
  const ChqLevel &C0 = lv[0];
  const int mz = (L.nz + 1) / 2;
  dim3 block(64, 4), grid((mz + 63) / 64, (L.ny + 3) / 4, L.nx);
  if (vec_ok(L))
    launch_pdl(k_chq_add_correction<true>, grid, block, 0, s, x, (long long)L.xstride, (long long)L.ystride, L.nx,
               L.ny, L.nz, C0.u[0], C0.u[1], C0.rz);
  else
    launch_pdl(k_chq_add_correction<false>, grid, block, 0, s, x, (long long)L.xstride, (long long)L.ystride, L.nx,
               L.ny, L.nz, C0.u[0], C0.u[1], C0.rz);
  return check_launch("k_chq_add_correction");
}

}  // namespace ocub
