// Device code of the red/black split ("chequer") FP32 multigrid levels, shared by the level
// kernels of the refinement solver (ir_chequer.cu) and the persistent ensemble
// (ensemble_persistent.cu): boundary and coefficient records, the per-item bodies of a colour
// sweep, a residual restriction and a prolongation, and the single-block schedule of the small
// levels staged in shared memory.  The layout is described in ir_chequer.h.
#pragma once

#include <cstdlib>

#include "ir_chequer.h"

namespace ocub {
namespace chq {
// internal linkage: every translation unit that includes this header gets its own copies
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

// Division of a non-negative int by a run-time constant d: a shift and a mask when d is a power
// of two, else a multiply-high by a precomputed magic number (Granlund and Montgomery, "Division
// by invariant integers using multiplication", 1994: l = ceil(log2 d),
// m = floor(2^32 (2^l - d) / d) + 1, q = (umulhi(m, t) + t) >> l, exact for 0 <= t < 2^31).
struct FDiv {
  int d, sh;    // divisor; log2 d when a power of two, else -1
  unsigned m;   // magic multiplier
  int l;        // ceil(log2 d)
};

inline FDiv make_fdiv(int d) {
  FDiv f;
  f.d = d;
  f.l = 0;
  while ((1LL << f.l) < d) f.l++;
  f.sh = ((1LL << f.l) == d) ? f.l : -1;
  f.m = (unsigned)((((unsigned long long)1 << 32) * (((unsigned long long)1 << f.l) - d)) / d + 1);
  return f;
}

__device__ __forceinline__ void split(const FDiv &f, int t, int &quot, int &rem) {
  if (f.sh >= 0) {
    quot = t >> f.sh;
    rem = t & (f.d - 1);
  } else {
    quot = (int)(((unsigned long long)__umulhi((unsigned)t, f.m) + (unsigned)t) >> f.l);
    rem = t - quot * f.d;
  }
}

struct ChqG {
  float *u0, *u1, *b0, *b1;
  int nx, ny, nz, rz;
  FDiv fq, fy;  // division by rz/4 (float4 groups per row) and by ny
};

inline int log2_exact(int v) {
  if (v <= 0 || (v & (v - 1))) return -1;
  int s = 0;
  while ((1 << s) < v) s++;
  return s;
}

inline float sgn_of(const ocu_bc &b) {
  if (b.type == OCU_BC_NEUMANN) return 1.f;
  if (b.type == OCU_BC_DIRICHELET) return -1.f;
  return 0.f;
}

// Loads of the level arrays: NC = true through the read-only path (the level kernels, where no
// launch writes what it reads that way); false plain loads (a persistent kernel whose blocks
// read, after a barrier, what they wrote earlier in the same launch).
template <bool NC>
__device__ __forceinline__ float ld1(const float *p) {
  if constexpr (NC) return __ldg(p);
  else return *p;
}
template <bool NC>
__device__ __forceinline__ float2 ld2(const float *p) {
  if constexpr (NC) return __ldg(reinterpret_cast<const float2 *>(p));
  else return *reinterpret_cast<const float2 *>(p);
}
template <bool NC>
__device__ __forceinline__ float4 ld4(const float *p) {
  if constexpr (NC) return __ldg(reinterpret_cast<const float4 *>(p));
  else return *reinterpret_cast<const float4 *>(p);
}
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
template <bool NC>
__device__ __forceinline__ void chq_relax_item(const ChqG &g, const ChqK &k, const ChqBC &bc, int color, int t) {
  int row, q, i, j;
  split(g.fq, t, row, q);
  split(g.fy, row, i, j);
  const int p = (i + j + color) & 1;
  const float *__restrict__ o = color ? g.u0 : g.u1;
  float *__restrict__ u = color ? g.u1 : g.u0;
  const float *__restrict__ bb = color ? g.b1 : g.b0;
  const long long rs = (long long)row * g.rz;
  const long long base = rs + 4 * q;
  const long long xs = (long long)g.ny * g.rz;
  const float4 U = *reinterpret_cast<const float4 *>(u + base);
  const float4 B = *reinterpret_cast<const float4 *>(bb + base);
  const float4 O = ld4<NC>(o + base);
  float4 XM, XP, YM, YP;
  if (i > 0) XM = ld4<NC>(o + base - xs);
  else XM = bc.px ? ld4<NC>(o + base + (long long)(g.nx - 1) * xs) : scale4(U, bc.sxn);
  if (i < g.nx - 1) XP = ld4<NC>(o + base + xs);
  else XP = bc.px ? ld4<NC>(o + base - (long long)(g.nx - 1) * xs) : scale4(U, bc.sxp);
  if (j > 0) YM = ld4<NC>(o + base - g.rz);
  else YM = bc.py ? ld4<NC>(o + base + (long long)(g.ny - 1) * g.rz) : scale4(U, bc.syn);
  if (j < g.ny - 1) YP = ld4<NC>(o + base + g.rz);
  else YP = bc.py ? ld4<NC>(o + base - (long long)(g.ny - 1) * g.rz) : scale4(U, bc.syp);
  float oprev = 0.f, onext = 0.f;
  if (p == 0) {
    if (q > 0) oprev = ld1<NC>(o + base - 1);
  } else if (8 * q + 8 < g.nz) {
    onext = ld1<NC>(o + base + 4);
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
        zm = bc.pz ? ld1<NC>(o + rs + (g.nz / 2 - 1)) : bc.szn * uo[e];
        mod += bc.mzn;
      }
      if (kk == g.nz - 1) {
        zp = bc.pz ? ld1<NC>(o + rs) : bc.szp * uo[e];
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
template <bool NC>
__device__ __forceinline__ void load4(const FRow &r, int m2, float v[4]) {
  const float2 A = ld2<NC>(r.a + m2);
  const float2 O = ld2<NC>(r.o + m2);
  v[0] = A.x; v[1] = O.x; v[2] = A.y; v[3] = O.y;
}

// Residual of the sixteen children of a coarse pair (coarse cells K = 2m', 2m' + 1 of coarse
// row (I, J)), restricted (the mean of each cell's eight) into the coarse right-hand side; the
// coarse pair's u is zeroed (the next V-cycle leg starts from zero).  All lanes of a warp share
// (I, J), so every row and boundary decision is uniform across the warp.
// ZU: the fine u is zero (a correction solve's first descent), so only b is read: with every u
// term zero residual_cell returns b itself (each product is +0, and b - (+0) == b, signed
// zeros included), so the sums are the general path's, bit for bit.
template <bool NC, bool ZU = false>
__device__ __forceinline__ void chq_restrict_item(const ChqG &f, const ChqG &c, const ChqK &k, const ChqBC &bc,
                                                  const FDiv &fcm, int t) {
  int r, mp, I, J;
  split(fcm, t, r, mp);
  split(c.fy, r, I, J);
  const int x0 = 2 * I, y0 = 2 * J, m2 = 2 * mp;
  const bool second = 2 * mp + 1 < c.nz;  // coarse K = 2m' + 1 exists
  const long long cid = ((long long)I * c.ny + J) * c.rz + mp;
  const bool sc = (I + J) & 1;  // coarse row parity: K = 2m' is colour sc entry m', K = 2m' + 1 colour sc^1
  if (ZU) {
    float sum[2] = {0.f, 0.f};
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 2; b++) {
        float bv[4];
        load4<NC>(fine_row(f.b0, f.b1, f, x0 + a, y0 + b), m2, bv);
#pragma unroll
        for (int e = 0; e < 4; e++) sum[e >> 1] += bv[e];
      }
    (sc ? c.b1 : c.b0)[cid] = 0.125f * sum[0];
    (sc ? c.u1 : c.u0)[cid] = 0.f;
    if (second) {
      (sc ? c.b0 : c.b1)[cid] = 0.125f * sum[1];
      (sc ? c.u0 : c.u1)[cid] = 0.f;
    }
    return;
  }
  float u[2][2][6], bv[2][2][4];           // u[a][b][1 + e], e = -1..4
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++) {
      const FRow R = fine_row(f.u0, f.u1, f, x0 + a, y0 + b);
      const FRow RB = fine_row(f.b0, f.b1, f, x0 + a, y0 + b);
      float v[4];
      load4<NC>(R, m2, v);
#pragma unroll
      for (int e = 0; e < 4; e++) u[a][b][1 + e] = v[e];
      load4<NC>(RB, m2, bv[a][b]);
      // k = 4m' - 1: colour s^1 entry 2m' - 1; k = 4m' + 4: colour s entry 2m' + 2
      if (mp > 0) u[a][b][0] = ld1<NC>(R.o + m2 - 1);
      else u[a][b][0] = bc.pz ? ld1<NC>(R.o + f.nz / 2 - 1) : bc.szn * u[a][b][1];
      if (4 * mp + 4 < f.nz) u[a][b][5] = ld1<NC>(R.a + m2 + 2);
      else u[a][b][5] = bc.pz ? ld1<NC>(R.a) : bc.szp * u[a][b][4];
      // an odd coarse row ends on K = 2m': the fine row ends on k = 4m' + 1 (its z+ neighbour is
      // the boundary value); k = 4m' + 2, 4m' + 3 are padding and their residuals unused
      if (!second) u[a][b][3] = bc.szp * u[a][b][2];
    }
  // rows around the 2x2 block of child rows: xo[side][b][e], yo[a][side][e]
  float xo[2][2][4], yo[2][2][4];
#pragma unroll
  for (int b = 0; b < 2; b++) {
    const int y = y0 + b;
    if (x0 > 0 || bc.px) load4<NC>(fine_row(f.u0, f.u1, f, x0 > 0 ? x0 - 1 : f.nx - 1, y), m2, xo[0][b]);
    else
#pragma unroll
      for (int e = 0; e < 4; e++) xo[0][b][e] = bc.sxn * u[0][b][1 + e];
    if (x0 + 2 < f.nx || bc.px) load4<NC>(fine_row(f.u0, f.u1, f, x0 + 2 < f.nx ? x0 + 2 : 0, y), m2, xo[1][b]);
    else
#pragma unroll
      for (int e = 0; e < 4; e++) xo[1][b][e] = bc.sxp * u[1][b][1 + e];
  }
#pragma unroll
  for (int a = 0; a < 2; a++) {
    const int x = x0 + a;
    if (y0 > 0 || bc.py) load4<NC>(fine_row(f.u0, f.u1, f, x, y0 > 0 ? y0 - 1 : f.ny - 1), m2, yo[a][0]);
    else
#pragma unroll
      for (int e = 0; e < 4; e++) yo[a][0][e] = bc.syn * u[a][0][1 + e];
    if (y0 + 2 < f.ny || bc.py) load4<NC>(fine_row(f.u0, f.u1, f, x, y0 + 2 < f.ny ? y0 + 2 : 0), m2, yo[a][1]);
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
  (sc ? c.b1 : c.b0)[cid] = 0.125f * sum[0];
  (sc ? c.u1 : c.u0)[cid] = 0.f;
  if (second) {
    (sc ? c.b0 : c.b1)[cid] = 0.125f * sum[1];
    (sc ? c.u0 : c.u1)[cid] = 0.f;
  }
}


// Where a prolongation's result goes.  ADD: added to the fine u.  ASSIGN: the fine u is zero
// (the first ascent of a correction solve) and is not read; the result is fma(p, 1/64, 0), the
// ADD result for a zero fine u, bit for bit.  X64 / X64V: the fine u (the refinement's FP32
// correction e) is read, e + p/64 is formed as in ADD and added in double to the FP64 solution
// x instead of being stored (the correction solve's last step fused with x += e); X64V moves
// x as 16-byte double pairs (k even, pairs 16-byte aligned).
enum { CHQ_P_ADD = 0, CHQ_P_ASSIGN = 1, CHQ_P_X64 = 2, CHQ_P_X64V = 3 };

struct ChqX {
  double *x;       // the FP64 level-0 grid at its interior origin
  long long xs, ys;
};

// Trilinear prolongation (weights 27, 9, 3, 1 / 64) of a coarse pair (K = 2m', 2m' + 1 of coarse
// row (I, J)) into its sixteen children, added to the fine u (MODE: see above).  Coarse values
// outside the domain follow the homogeneous rules axis by axis (a corner is the product of the
// face signs times the cell).  Rows are warp-uniform; the eight fine float2 pairs are loaded
// before the first store.
template <bool NC, int MODE = CHQ_P_ADD>
__device__ __forceinline__ void chq_prolong_item(const ChqG &c, const ChqG &f, const ChqBC &bc, const FDiv &fcm,
                                                 int t, ChqX X = ChqX{nullptr, 0, 0}) {
  int r, mp, I, J;
  split(fcm, t, r, mp);
  split(c.fy, r, I, J);
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
      const float v0 = ld1<NC>(R.a + mp);
      const float v1 = second ? ld1<NC>(R.o + mp) : (bc.pz ? ld1<NC>(R.a) : bc.szp * v0);
      float vm, vp;
      if (mp > 0) vm = ld1<NC>(R.o + mp - 1);
      else vm = bc.pz ? ld1<NC>(R.o + c.nz / 2 - 1) : bc.szn * v0;
      if (K0 + 2 < c.nz) vp = ld1<NC>(R.a + mp + 1);
      else vp = bc.pz ? ld1<NC>(R.a) : bc.szp * v1;
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
      if (MODE == CHQ_P_ASSIGN) {
        fa[a][b] = make_float2(0.f, 0.f);
        fo[a][b] = make_float2(0.f, 0.f);
      } else {
        fa[a][b] = *dA[a][b];
        fo[a][b] = *dO[a][b];
      }
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
      if (MODE == CHQ_P_ADD || MODE == CHQ_P_ASSIGN) {
        *dA[a][b] = A;
        *dO[a][b] = O;
      } else {
        // fine k = 4m' + e: e = 0 A.x, 1 O.x, 2 A.y, 3 O.y (k = 4m' + 2, + 3 only with `second`)
        double *px = X.x + (long long)(2 * I + a) * X.xs + (long long)(2 * J + b) * X.ys + 4 * mp;
        if (MODE == CHQ_P_X64V) {
          double2 *p2 = reinterpret_cast<double2 *>(px);
          double2 v = p2[0];
          v.x = v.x + (double)A.x;
          v.y = v.y + (double)O.x;
          p2[0] = v;
          if (second) {
            double2 w = p2[1];
            w.x = w.x + (double)A.y;
            w.y = w.y + (double)O.y;
            p2[1] = w;
          }
        } else {
          px[0] = px[0] + (double)A.x;
          px[1] = px[1] + (double)O.x;
          if (second) {
            px[2] = px[2] + (double)A.y;
            px[3] = px[3] + (double)O.y;
          }
        }
      }
    }
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

// The tail schedule of one launch (FMG from level s's right-hand side, or one V-cycle), on the
// level table lv in shared memory and the staging area sm; block-wide.
__device__ __forceinline__ void chq_tail_run(const ChqTail &T, const SLv *lv, float *sm) {
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


inline ChqBC make_bc(const ocu_bc_set &bc, double fx, double fy, double fz) {
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

inline ChqK make_k(double h, double fx, double fy, double fz, double omega) {
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

inline ChqG make_g(const ChqLevel &l) {
  ChqG g;
  g.u0 = l.u[0]; g.u1 = l.u[1]; g.b0 = l.b[0]; g.b1 = l.b[1];
  g.nx = l.nx; g.ny = l.ny; g.nz = l.nz; g.rz = l.rz;
  g.fq = make_fdiv(l.rz / 4);
  g.fy = make_fdiv(l.ny);
  return g;
}

inline int round4(int v) { return (v + 3) & ~3; }

// Shared memory of a level in the single-CTA tail: its four colour arrays.
inline size_t level_smem(const std::array<int, 3> &d) {
  return (size_t)4 * d[0] * d[1] * round4((d[2] + 1) / 2) * sizeof(float);
}

// the tail's residual scratch: two colour arrays of its largest restricted level
inline size_t scratch_smem(const std::array<int, 3> &d) { return level_smem(d) / 2; }

// Largest shared-memory footprint of the tail kernel (opt-in above 48 KB).
constexpr size_t kTailSmemCap = 200 * 1024;
// Levels with at most this many cells join the single-CTA tail (OCU_B200_CHQ_TAIL overrides;
// the coarsest level always runs there).  Measured at 256^3 (refinement solve, one box): 3.82 ms
// with only the coarsest level (4^3) in the tail, 3.75 ms with 8^3 too, 3.78 ms with 16^3 too --
// a tail phase over a 16^3 level costs about what a launch with programmatic dependencies does.
constexpr long long kChqTailCells = 512;

inline long long tail_cells_setting() {
  const char *e = std::getenv("OCU_B200_CHQ_TAIL");
  return e ? std::atoll(e) : kChqTailCells;
}

// First level of the single-CTA tail: the largest run of coarse levels, each with at most
// tail_cells cells, whose arrays fit the shared-memory cap (at least the coarsest level).
inline int tail_first(const std::vector<std::array<int, 3>> &dims, long long tail_cells) {
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

}  // namespace
}  // namespace chq
}  // namespace ocub
